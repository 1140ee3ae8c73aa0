"""FP32-bulk path (reconstruction, limiter and fluxes in single precision;
geometry, face velocity, accumulation and the cell update in double): its
error against the FP64 oracle, stated per conserved variable, and exact
conservation."""
import numpy as np
import pytest

from common import setup_case

pytestmark = pytest.mark.gpu

# Relative L1 error bound per conserved variable after the steps below
# (sum |fp32 - oracle| / sum |oracle|; a magnetic component against the L1
# norm of the whole field, since one component can start at zero): single
# precision carries ~1e-7 relative error into each flux, and the measured
# errors are 1e-9 to 1e-6.
RTOL_L1_FP32 = 1e-5


def run(problem, nside, nsteps, precision):
    import fvmhd3d_b200 as F
    m, W = setup_case(nside, problem, seed=nside, noise=0.0)
    s = F.System(precision=precision)
    s.set_mesh(m)
    s.init_problem(W)
    for _ in range(nsteps):
        s.step(shared=True)
    return m, W, s


def oracle(m, W, nsteps):
    from oracle.pyoracle import OracleSystem
    o = OracleSystem()
    o.set_mesh(m)
    o.init_problem(W)
    for _ in range(nsteps):
        o.step(shared=True)
    return o


@pytest.mark.parametrize("problem,nside,nsteps", [("blast", 24, 12), ("orszag_tang", 20, 10)])
def test_fp32_error_vs_fp64_oracle(problem, nside, nsteps):
    import fvmhd3d_b200 as F
    m, W, s = run(problem, nside, nsteps, F.FVM_PREC_FP32)
    o = oracle(m, W, nsteps)
    a, b = s.get_state()["U"], o.get_state()["U"]
    den = np.abs(b).sum(axis=0)
    den[5:8] = np.sqrt((b[:, 5:8] ** 2).sum(axis=1)).sum()
    l1 = np.abs(a - b).sum(axis=0) / np.maximum(den, 1e-300)
    print(problem, "rel L1 per conserved variable:", " ".join("%.2e" % x for x in l1))
    for k in (0, 1, 2, 3, 4, 5, 6, 7):  # mass, momentum, energy, magnetic flux
        assert l1[k] <= RTOL_L1_FP32, (k, l1[k])
    assert np.isfinite(a).all()


def test_fp32_conserves_exactly():
    import fvmhd3d_b200 as F
    m, W, s = run("blast", 24, 0, F.FVM_PREC_FP32)
    U0 = s.get_state()["U"].sum(axis=0)
    for _ in range(10):
        s.step(shared=True)
    U = s.get_state()["U"]
    scale = np.abs(U).sum(axis=0)
    for k in (0, 1, 2, 3, 4):
        assert abs(U.sum(axis=0)[k] - U0[k]) <= 1e-13 * scale[k], k


def test_fp32_state_roundtrip():
    import fvmhd3d_b200 as F
    m, W, s = run("alfven", 8, 2, F.FVM_PREC_FP32)
    st = s.get_state()
    s.set_state(vel=st["vel"], tlast=st["tlast"], tend=st["tend"], rung=st["rung"], U=st["U"], dU=st["dU"],
                wrec=st["wrec"], tsys_ticks=s.tsys_ticks)
    st2 = s.get_state()
    for k in st:
        assert np.array_equal(st[k], st2[k]), k
