"""The order parameters without device allocation, checked against the
context-based entry point.

``gcr_order_params_noalloc`` is for callers that cannot allocate device
memory (an analysis hook sampling while other work is queued, since cudaFree
waits for the whole device; an application that owns all device memory
through its own pool).  It must give what ``gcr_order_params`` gives, call
after call, although its scratch is one static device array shared by every
call, and a call with bad chain ids must not leave anything that changes the
next call's result.  This file is collected last so that a run stopping at
the first failure has run every other test first; it also passes alone in a
fresh process.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import _lib  # noqa: E402
from gliding_collective_rotation_b200.engine import Engine, SystemParams, SystemState  # noqa: E402
from gliding_collective_rotation_b200.engine import wca_params as make_WCA_params  # noqa: E402


def _system(n_chains, chain_length, seed):
    rng = np.random.default_rng(seed)
    n = n_chains * chain_length
    # chains with a common drift plus noise, so that P and S are non-trivial
    base = rng.uniform(0, 2 * np.pi, size=n_chains)
    ang = np.repeat(base, chain_length) + 0.3 * rng.standard_normal(n)
    tan = np.stack([np.cos(ang), np.sin(ang)], axis=1)
    pos = rng.uniform(0, 40.0, size=(n, 2))
    chain = np.repeat(np.arange(n_chains), chain_length)
    return pos, tan, chain


def _params():
    return SystemParams(L=40.0, spring_params=np.array([100.0, 20.0, 0.0, 0.0, 1.0, 0.1]),
                        wca_params=make_WCA_params(1.0, 1.0, 0.0, 1.0), active_params=np.array([1.0, 0.0, 0.0]),
                        D=0.01, Dr=0.0075, radius=1.0, n_nearby=4)


def _noalloc(state, precision_code):
    out = (C.c_double * 3)()
    lib = _lib.load()
    torch.cuda.synchronize()
    rc = lib.gcr_order_params_noalloc(2, precision_code, C.c_void_p(state.tangent.data_ptr()),
                                      C.c_void_p(state.chain_id.data_ptr()), state.n, state.n_chains, out,
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc)
    return np.array(out[:])


@pytest.mark.parametrize("precision,code", [("fp64", _lib.GCR_FP64), ("mixed", _lib.GCR_MIXED)])
def test_noalloc_matches_context_entry_point_twice(precision, code):
    """Two calls in a row on different systems: each equals the context-based
    result within the tolerance of the other order-parameter tests (1e-12);
    the second call is not disturbed by what the first left in the scratch."""
    for call, (nc, cl, seed) in enumerate([(500, 10, 1), (300, 7, 2)]):
        pos, tan, chain = _system(nc, cl, seed)
        with Engine(2, precision, bead_capacity=len(pos), system_capacity=1, cell_capacity=4 * len(pos)) as eng:
            st = SystemState.from_host(pos, tan, chain, np.full(nc, 0.5), _params(), precision=precision)
            slot = eng.admit(st)
            want = eng.order_params(slot)
            got = _noalloc(st, code)
            assert np.allclose(got, want, rtol=1e-12, atol=1e-12), (call, got, want)
            # repeating the call on the same data gives the same numbers
            assert np.array_equal(_noalloc(st, code), got)


@pytest.mark.parametrize("bad_ids", [[0, 0, 2, 2], [1, 1, 2, 2], [0, 1, 1, 0], [0, 0, 1, 1]])
def test_noalloc_rejects_bad_chain_ids_and_the_next_call_is_clean(bad_ids):
    """Chain ids that skip a chain, do not start at 0, step back, or end
    before n_chains - 1 (here n_chains = 3) are refused with GCR_ERR_BAD_ARG;
    a valid call right after it still equals ``gcr_order_params`` (the error
    word and results are cleared by every call)."""
    lib = _lib.load()
    rng = np.random.default_rng(11)
    ang = rng.uniform(0, 2 * np.pi, 4)
    tan = torch.tensor(np.stack([np.cos(ang), np.sin(ang)], axis=1), dtype=torch.float64, device="cuda")
    chain = torch.tensor(bad_ids, dtype=torch.int32, device="cuda")
    out = (C.c_double * 3)()
    torch.cuda.synchronize()
    rc = lib.gcr_order_params_noalloc(2, _lib.GCR_FP64, C.c_void_p(tan.data_ptr()), C.c_void_p(chain.data_ptr()),
                                      4, 3, out, None)
    assert rc == -1  # GCR_ERR_BAD_ARG
    assert b"chain ids" in lib.gcr_last_error()
    pos, tan_ok, chain_ok = _system(40, 6, 3)
    with Engine(2, "fp64", bead_capacity=len(pos), system_capacity=1, cell_capacity=4 * len(pos)) as eng:
        st = SystemState.from_host(pos, tan_ok, chain_ok, np.full(40, 0.5), _params(), precision="fp64")
        slot = eng.admit(st)
        want = eng.order_params(slot)
        got = _noalloc(st, _lib.GCR_FP64)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12), (got, want)


def test_noalloc_rejects_more_chains_than_its_scratch_holds():
    lib = _lib.load()
    n_chains = 262144 + 1
    tan = torch.zeros((n_chains, 2), dtype=torch.float64, device="cuda")
    chain = torch.arange(n_chains, dtype=torch.int32, device="cuda")
    out = (C.c_double * 3)()
    rc = lib.gcr_order_params_noalloc(2, _lib.GCR_FP64, C.c_void_p(tan.data_ptr()), C.c_void_p(chain.data_ptr()),
                                      n_chains, n_chains, out, None)
    assert rc == -6
    assert b"GCR_NOALLOC_MAX_CHAINS" in lib.gcr_last_error()
