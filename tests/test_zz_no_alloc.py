"""asr_cf_eval_noalloc (fractions staged through a static device array) against asr_cf_eval, through the C ABI."""
import ctypes as C

import numpy as np
import pytest

from asr_b200 import _lib
from asr_b200.augcls import default_context

pytestmark = pytest.mark.gpu


def _chains(seed, ld, nchain, nz):
    rng = np.random.default_rng(seed)
    a = np.asfortranarray(rng.uniform(-0.5, 0.5, (ld, nchain)) + 1j * rng.uniform(-0.05, 0.0, (ld, nchain)))
    b = np.asfortranarray(rng.uniform(0.2, 0.5, (ld, nchain)) + 1j * rng.uniform(-0.03, 0.03, (ld, nchain)))
    m = rng.integers(4, ld + 1, nchain).astype(np.int32)
    z = np.asfortranarray(rng.uniform(-0.8, 0.8, (nz, nchain)) + 1j * rng.uniform(0.005, 0.2, (nz, nchain)))
    return a, b, m, z


def _pd(x):
    return x.ctypes.data_as(C.POINTER(C.c_double))


def _run(fn, ctx, a, b, m, z, tail):
    ld, nc = a.shape
    nz = z.shape[0]
    g = np.zeros((nz, nc), np.complex128, order="F")
    nf = C.c_int64(-1)
    args = [ctx.h, _pd(a), _pd(b), m.ctypes.data_as(C.POINTER(C.c_int)), ld, nc, _pd(z), nz, _lib.TAILS[tail], _pd(g)]
    if fn == "asr_cf_eval":
        args.append(None)   # no edges
    args.append(C.byref(nf))
    _lib.check(getattr(_lib.lib(), fn)(*args))
    return g, nf.value


@pytest.mark.parametrize("tail", ["hull", "avg2", "bp", "none"])
def test_noalloc_matches_cf_eval_on_two_calls_in_a_row(tail):
    ctx = default_context()
    for seed, (ld, nc, nz) in ((1, (24, 40, 33)), (2, (16, 7, 200))):
        a, b, m, z = _chains(seed, ld, nc, nz)
        g_ref, nf_ref = _run("asr_cf_eval", ctx, a, b, m, z, tail)
        g_new, nf_new = _run("asr_cf_eval_noalloc", ctx, a, b, m, z, tail)
        assert np.max(np.abs(g_new - g_ref) / np.abs(g_ref)) < 1e-13
        assert nf_new == nf_ref


def test_noalloc_rejects_operands_above_the_scratch():
    ctx = default_context()
    ld, nc = 64, 4096   # a and b alone need 2 x 64 x 4096 x 16 B = 8 MiB
    a = np.zeros((ld, nc), np.complex128, order="F")
    b = np.zeros((ld, nc), np.complex128, order="F")
    m = np.full(nc, 4, np.int32)
    z = np.full((1, nc), 0.1j, np.complex128, order="F")
    g = np.zeros((1, nc), np.complex128, order="F")
    rc = _lib.lib().asr_cf_eval_noalloc(ctx.h, _pd(a), _pd(b), m.ctypes.data_as(C.POINTER(C.c_int)), ld, nc, _pd(z), 1,
                                       _lib.TAILS["hull"], _pd(g), None)
    assert rc == _lib.ASR_EINVAL
    assert "static scratch" in _lib.last_error()
