"""fvm_step_host: one step on host-owned state with the copies of U and dU
overlapped with the stage kernels.  It must give the bits of fvm_set_state +
fvm_step + fvm_get_state, step after step."""
import numpy as np
import pytest

from common import golden_params, load_golden, setup_case
from test_gpu_parity import gpu_system

pytestmark = pytest.mark.gpu

KEYS = ("vel", "tlast", "tend", "rung", "U", "dU", "wrec")


def host_state(s):
    st = s.get_state()
    out = {}
    for k, t, w in s.STATE_ARRAYS:
        out[k] = np.ascontiguousarray(np.asarray(st[k]).reshape(-1) if w == 1 else st[k], t)
    return out


def run_both(a, b, nsteps, shared):
    """a: set_state, step, get_state each step; b: step_host on its own copy."""
    ha, hb = host_state(a), host_state(b)
    for _ in range(nsteps):
        ticks = a.tsys_ticks
        a.set_state(tsys_ticks=ticks, **ha)
        na = a.step(shared=shared)
        sa = a.get_state()
        for k in KEYS:
            ha[k] = np.ascontiguousarray(np.asarray(sa[k]).reshape(ha[k].shape), ha[k].dtype)
        nb = b.step_host(hb, shared=shared, tsys_ticks=ticks)
        assert na == nb
        for k in KEYS:
            assert np.array_equal(ha[k], hb[k]), k
        assert a.tsys_ticks == b.tsys_ticks and a.time == b.time


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_step_host_gives_the_set_step_get_bits(precision):
    import fvmhd3d_b200 as F
    prec = F.FVM_PREC_FP32 if precision == "fp32" else F.FVM_PREC_FP64
    m, W = setup_case(12, "blast", seed=3, noise=0.02)
    a, b = gpu_system(m, W, precision=prec), gpu_system(m, W, precision=prec)
    run_both(a, b, 4, shared=True)


def test_step_host_individual_timesteps_on_the_disk_golden():
    m, z = load_golden("ref_disk4k_individual.npz")
    kw = golden_params(z)
    a = gpu_system(m, z["W"], bnd=z.get("bnd"), **kw)
    b = gpu_system(m, z["W"], bnd=z.get("bnd"), **kw)
    run_both(a, b, 6, shared=False)


def test_step_host_rejects_a_rung_out_of_range_before_uploading():
    import fvmhd3d_b200 as F
    m, W = setup_case(8, "alfven", seed=2, noise=0.0)
    s = gpu_system(m, W)
    h = host_state(s)
    before = s.get_state()
    bad = {k: v.copy() for k, v in h.items()}
    bad["rung"][5] = 40
    bad["U"][:] = 0.0
    with pytest.raises(F.FvmError):
        s.step_host(bad, shared=True)
    after = s.get_state()
    for k in before:
        assert np.array_equal(before[k], after[k]), k
    with pytest.raises(ValueError):
        s.step_host({**h, "U": h["U"][:10]}, shared=True)


def test_remesh_every_step_keeps_the_bits():
    """The flow of a host that rebuilds its mesh every step: fvm_set_mesh,
    fvm_set_positions, then the state it keeps (fvm_step_host).  Reinstalling
    the same mesh each step gives the bits of steps on one installed mesh."""
    m, z = load_golden("ref_disk4k_individual.npz")
    kw = golden_params(z)
    bnd = z.get("bnd")
    a = gpu_system(m, z["W"], bnd=bnd, **kw)
    b = gpu_system(m, z["W"], bnd=bnd, **kw)
    hb = host_state(b)
    for _ in range(5):
        a.step(shared=False)
        ticks = b.tsys_ticks
        b.set_mesh(m)
        b.set_positions(m.pos, bnd)
        b.step_host(hb, shared=False, tsys_ticks=ticks)
    sa = a.get_state()
    for k, t, w in b.STATE_ARRAYS:
        assert np.array_equal(np.asarray(sa[k], t).reshape(hb[k].shape), hb[k]), k
    assert a.tsys_ticks == b.tsys_ticks


def test_a_new_mesh_needs_its_positions_before_a_state():
    import fvmhd3d_b200 as F
    m, W = setup_case(8, "alfven", seed=2, noise=0.0)
    s = gpu_system(m, W)
    h = host_state(s)
    s.set_mesh(m)
    with pytest.raises(F.FvmError):
        s.set_state(**h)
    with pytest.raises(F.FvmError):
        s.step_host(h, shared=True)
    s.set_positions(m.pos)
    s.set_state(**h)
    s.step(shared=True)
