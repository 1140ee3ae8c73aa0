"""The plain-C oracle (oracle/fvm_oracle.c) is pinned bit for bit to the
reference's own hot path: against the committed golden fixtures (made by
tests/golden/make_golden.py from the reference build) and, where the
reference build is present, against it live."""
import os

import numpy as np
import pytest

from common import GOLDEN_STEP_CASES, ORACLE_SO, REF_SO, golden_params, load_golden, setup_case
from oracle.pyoracle import OracleSystem, RefSystem

pytestmark = pytest.mark.skipif(not os.path.exists(ORACLE_SO), reason="oracle not built")


@pytest.mark.parametrize("name", GOLDEN_STEP_CASES)
def test_oracle_matches_golden_bitexact(name):
    m, z = load_golden(name)
    o = OracleSystem(**golden_params(z))
    o.set_mesh(m)
    o.init_problem(z["W"], bnd=z.get("bnd"))
    nact = [o.step(shared=bool(z["shared"])) for _ in range(int(z["nsteps"]))]
    assert nact == list(z["out_nactive"])
    st = o.get_state()
    for k in ("pos", "vel", "tlast", "tend", "rung", "U", "dU", "wrec"):
        assert np.array_equal(st[k], z["out_" + k]), k
    assert o.time == z["out_time"]


def test_oracle_flux_matches_golden_bitexact():
    m, _ = load_golden("ref_alfven4_shared.npz")
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_flux_kat.npz"))
    o = OracleSystem()
    psi, Bn, flux = o.compute_flux(z["wij"], z["Wi"], z["Wj"], z["jbnd"], z["normal"])
    assert np.array_equal(psi, z["psi"]) and np.array_equal(Bn, z["Bn"]) and np.array_equal(flux, z["flux"])


needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build absent")


@needs_ref
@pytest.mark.parametrize("nside,problem,shared,nsteps", [
    (6, "alfven", True, 4), (6, "orszag_tang", True, 3), (8, "blast", False, 10), (7, "alfven", False, 6)])
def test_oracle_vs_reference_live(nside, problem, shared, nsteps):
    m, W = setup_case(nside, problem, seed=nside + 20)
    r, o = RefSystem(), OracleSystem()
    for s in (r, o):
        s.set_mesh(m)
        s.init_problem(W)
    for _ in range(nsteps):
        a = r.step(shared=shared, snap=True)
        b = o.step(shared=shared, snap=True)
        assert a["nactive"] == b["nactive"]
        assert np.array_equal(a["active_faces"], b["active_faces"])
        act = o.get_state()["tlast"] == o.time
        for k in ("wrec_after_limiter", "U_after_update", "dU_after_update", "vel_after_pvel",
                  "rung_after_timestep", "wrec_after_update0", "rung_after_update0", "wrec_after_recon"):
            assert np.array_equal(a[k][act], b[k][act]), k
    sa, sb = r.get_state(), o.get_state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k


@needs_ref
def test_oracle_flux_vs_reference_live():
    rng = np.random.default_rng(3)
    nf = 512
    Wi = np.abs(rng.normal(1, 0.5, (nf, 10))) + 0.05
    Wj = np.abs(rng.normal(1, 0.5, (nf, 10))) + 0.05
    Wi[:, 1:4] = rng.normal(size=(nf, 3)); Wj[:, 5:8] = rng.normal(size=(nf, 3))
    nrm = rng.normal(size=(nf, 3)); nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wij = rng.normal(size=(nf, 3))
    jb = rng.choice([0, 1, 2, 3], nf).astype(np.int32)
    a = RefSystem().compute_flux(wij, Wi, Wj, jb, nrm)
    b = OracleSystem().compute_flux(wij, Wi, Wj, jb, nrm)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
