"""Incremental list building of partial steps (k_inc_* in csrc/fvm_device.cuh):
a step with few active cells builds its face flags, active-face list and
involved-cell list from the active cells' links instead of a pass over every
face and cell (MPI/iterate.cpp:58-113 selects the same sites).  The lists
hold the same faces and cells, so the steps must give the same bits as with
the pass over every face, eager or replayed, with the stage kernels or the
persistent rung kernel."""
import numpy as np
import pytest

from common import load_golden, golden_params, setup_case
from test_fused import same_bits
from test_gpu_parity import gpu_system

pytestmark = pytest.mark.gpu


def contrast_blast(nside, seed):
    """A blast with a 1e4 pressure contrast: the hot centre sits on the
    highest rungs, so many partial steps have few active cells."""
    m, W = setup_case(nside, "blast", seed=seed, noise=0.02)
    W = W.copy()
    r = np.linalg.norm(m.pos - 0.5, axis=1)
    W[r < 0.12, 4] *= 1e4
    return m, W


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_incremental_lists_give_the_meshwide_bits(precision):
    """Eager steps with the pass over every face against eager and replayed
    steps that build small steps' lists incrementally (the automatic bound)."""
    import fvmhd3d_b200 as F
    prec = F.FVM_PREC_FP32 if precision == "fp32" else F.FVM_PREC_FP64
    m, W = contrast_blast(14, 9)
    a, b, c = (gpu_system(m, W, precision=prec) for _ in range(3))
    a.set_list_building(0)
    counts = [a.step(shared=False) for _ in range(14)]
    assert [c.step(shared=False) for _ in range(14)] == counts
    cells, _ = b.run(14, shared=False)
    assert cells == sum(counts)
    assert a.incremental_steps == 0
    assert c.incremental_steps >= 3 and b.incremental_steps == c.incremental_steps
    same_bits(a, b)
    same_bits(a, c)


def test_incremental_lists_with_the_persistent_kernel():
    """Replayed steps with both device-side choices (list building, then
    the persistent rung kernel or the stage kernels): the bits of eager
    steps with neither."""
    m, W = contrast_blast(12, 4)
    a, b = gpu_system(m, W), gpu_system(m, W)
    a.set_list_building(0)
    b.set_fused(m.ncell // 3)
    for _ in range(12):
        a.step(shared=False)
    b.run(12, shared=False)
    assert b.incremental_steps >= 2 and b.fused_steps >= 1
    same_bits(a, b)


@pytest.mark.parametrize("name", ["ref_disk4k_individual.npz", "ref_disk4k_static_individual.npz"])
def test_incremental_lists_on_the_disk_golden(name):
    """The Keplerian disk with a sink (boundary cells, whose faces are active
    only from their non-boundary side): eager steps with the pass over every
    face against replayed steps with incremental lists at a threshold that
    some steps pass and some do not."""
    m, z = load_golden(name)
    kw = golden_params(z)
    a = gpu_system(m, z["W"], bnd=z.get("bnd"), **kw)
    b = gpu_system(m, z["W"], bnd=z.get("bnd"), **kw)
    a.set_list_building(0)
    b.set_list_building(2000)
    nsteps = int(z["nsteps"])
    counts = [a.step(shared=False) for _ in range(nsteps)]
    cells, _ = b.run(nsteps, shared=False)
    assert cells == sum(counts)
    assert 1 <= b.incremental_steps < nsteps
    same_bits(a, b)


def test_list_building_setting_rejects_bad_values():
    import fvmhd3d_b200 as F
    m, W = setup_case(8, "alfven", seed=2, noise=0.0)
    s = gpu_system(m, W)
    for bad in (-2, -100):
        with pytest.raises(F.FvmError):
            s.set_list_building(bad)
    s.set_list_building(-1)
    s.run(2, shared=True)  # global steps build no lists
    assert s.incremental_steps == 0


def test_incremental_lists_with_the_learned_flux():
    """Learned-flux mode on individual timesteps (deferring pass, network,
    finishing pass over the active-face list): the faces' slots follow the
    list's order, but each face's network row and flux are its own, so the
    incremental lists give the bits of the pass over every face."""
    import fvmhd3d_b200 as F
    from fvmhd3d_b200 import learned as L
    model = L.load_model()
    m, W = contrast_blast(12, 5)
    a = gpu_system(m, W, precision=F.FVM_PREC_FP32)
    b = gpu_system(m, W, precision=F.FVM_PREC_FP32)
    for s in (a, b):
        L.apply(s, model)
        s.set_flux_mode(1, judge=4, **L.GATE)
    a.set_list_building(0)
    for _ in range(10):
        assert a.step(shared=False) == b.step(shared=False)
    assert b.incremental_steps >= 2
    same_bits(a, b)
    sa, sb = a.learn_stats(), b.learn_stats()
    assert sa["deferred"] > 0
    for k in ("deferred", "fallback", "judged", "positivity_fallback"):  # counts (the error sums are atomics)
        assert sa[k] == sb[k], k
