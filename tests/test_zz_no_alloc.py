"""fvm_compute_flux_static, the flux entry point that stages its batch in a
fixed device array instead of allocating, against fvm_compute_flux through
the C-ABI: identical results on two calls in a row (different batches, the
second smaller, with and without boundary flags), and batches above the
capacity rejected before any GPU work."""
import ctypes
import os

import numpy as np
import pytest

from common import GOLDEN

pytestmark = pytest.mark.gpu


def face_batch(nf, seed):
    rng = np.random.default_rng(seed)
    Wi = np.zeros((nf, 10))
    Wj = np.zeros((nf, 10))
    for W in (Wi, Wj):
        W[:, 0] = rng.uniform(0.1, 3.0, nf)
        W[:, 1:4] = rng.normal(0, 1.0, (nf, 3))
        W[:, 4] = rng.uniform(0.05, 5.0, nf)
        W[:, 5:8] = rng.normal(0, 1.0, (nf, 3))
        W[:, 8] = rng.normal(0, 0.1, nf)
        W[:, 9] = rng.uniform(0.5, 2.0, nf)
    nrm = rng.normal(size=(nf, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wij = rng.normal(0, 1.0, (nf, 3))
    jbnd = rng.choice(np.array([0, 0, 0, 1, 2, 3], np.int32), nf).astype(np.int32)
    return wij, Wi, Wj, jbnd, nrm


def call(lib, h, name, wij, Wi, Wj, jbnd, nrm):
    nf = Wi.shape[0]
    psi, Bn, flux = np.full(nf, np.nan), np.full(nf, np.nan), np.full((nf, 10), np.nan)
    args = [np.ascontiguousarray(a) for a in (wij, Wi, Wj)]
    jb = None if jbnd is None else np.ascontiguousarray(jbnd, np.int32)
    p = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    rc = getattr(lib, name)(h, nf, *[p(a) for a in args], p(jb), p(np.ascontiguousarray(nrm)),
                            p(psi), p(Bn), p(flux))
    return rc, psi, Bn, flux


@pytest.fixture(scope="module")
def ctx():
    import fvmhd3d_b200 as F
    s = F.System()
    return s, s.L, s.h


def test_static_flux_matches_allocating_entry_on_consecutive_calls(ctx):
    s, lib, h = ctx
    cap = 16384
    batches = [face_batch(cap, 1), face_batch(1000, 2)]  # full capacity, then a smaller batch
    for jb_on in (True, False):
        for wij, Wi, Wj, jbnd, nrm in batches:
            jb = jbnd if jb_on else None
            rc0, *ref = call(lib, h, "fvm_compute_flux", wij, Wi, Wj, jb, nrm)
            rc1, *got = call(lib, h, "fvm_compute_flux_static", wij, Wi, Wj, jb, nrm)
            assert rc0 == 0 and rc1 == 0, (rc0, rc1, lib.fvm_last_error(h))
            for a, b in zip(got, ref):
                assert np.isfinite(a).all()
                assert np.array_equal(a, b)


def test_static_flux_matches_reference_golden(ctx):
    s, lib, h = ctx
    z = np.load(os.path.join(GOLDEN, "ref_flux_kat.npz"))
    rc, psi, Bn, flux = call(lib, h, "fvm_compute_flux_static", z["wij"], z["Wi"], z["Wj"], z["jbnd"], z["normal"])
    assert rc == 0
    for a, b in ((psi, z["psi"]), (Bn, z["Bn"]), (flux, z["flux"])):
        den = np.abs(b).max(axis=0)
        assert (np.abs(a - b).max(axis=0) <= 1e-12 * np.where(den > 0, den, 1.0)).all()


def test_static_flux_rejects_batches_above_capacity(ctx):
    s, lib, h = ctx
    wij, Wi, Wj, jbnd, nrm = face_batch(16385, 3)
    rc, psi, _, _ = call(lib, h, "fvm_compute_flux_static", wij, Wi, Wj, jbnd, nrm)
    assert rc == -5  # FVM_ERANGE
    assert b"exceeds the static staging capacity of 16384 faces" in lib.fvm_last_error(h)
    assert np.isnan(psi).all()  # nothing written
