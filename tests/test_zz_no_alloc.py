"""btam_mf_eval_noalloc: the evaluation entry point that allocates no device
memory, for callers that may not call cudaMalloc themselves (their device
memory is owned by another allocator, or an allocation's implicit
synchronisation is not allowed).  It must give the same results as the
ordinary entry point, call after call, although every call reuses the same
fixed scratch inside the library.

This file is named to be collected last, so that a run stopping at the first
failure has already run every other test; it also passes alone in a fresh
process (it sets up everything it uses)."""
import numpy as np
import pytest

import btam
from btam import lattice

pytestmark = pytest.mark.gpu


def device_inputs(S, s, torch):
    """The all-sites input arrays of btam_mf_eval_noalloc, in caller-owned
    device memory (the caller allocates; the entry point does not)."""
    n = len(s["x"])
    qg, og, _ = S.ghosts()
    owner = np.concatenate([np.arange(n), og]).astype(np.int32)
    q_all = np.concatenate([s["q"], qg])
    pos4 = np.column_stack([q_all, s["sigma"][owner]])
    xb = np.column_stack([s["x"][owner], s["beta"][owner]])
    code = (s["species"][owner] == 1).astype(np.int32)
    offs, idx = S.neighbors()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return dict(pos4=dev(pos4), xb=dev(xb), code=dev(code), owner=dev(owner),
                gamma=dev(s["gamma"]), offs=dev(offs), idx=dev(idx))


def call_noalloc(tables, prec, n, inp, torch):
    out = dict(V0=torch.zeros(n, dtype=torch.float64, device="cuda"),
               Rq=torch.zeros((n, 3), dtype=torch.float64, device="cuda"),
               Rs=torch.zeros(n, dtype=torch.float64, device="cuda"),
               Rx=torch.zeros(n, dtype=torch.float64, device="cuda"),
               totals=torch.zeros(4, dtype=torch.float64, device="cuda"))
    p = lambda t: t.data_ptr()
    code = btam.lib().btam_mf_eval_noalloc(
        tables.handle, prec, n, p(inp["pos4"]), p(inp["xb"]), p(inp["code"]),
        p(inp["owner"]), p(inp["gamma"]), p(inp["offs"]), p(inp["idx"]), p(out["V0"]),
        p(out["Rq"]), p(out["Rs"]), p(out["Rx"]), p(out["totals"]),
        torch.cuda.current_stream().cuda_stream)
    assert code == 0, btam.STATUS.get(code, code)
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("prec", [btam.FP64, btam.FP32C])
def test_noalloc_matches_allocating_entry_point(gpu_tables, prec):
    torch = pytest.importorskip("torch")
    s = lattice.config1(seed=7)
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    ref = S.evaluate(prec)
    n = len(s["x"])
    inp = device_inputs(S, s, torch)
    # tolerances of the parity tests: FP64 1e-10 relative, FP32C 1e-6 relative
    # energy and 1e-5 on residual components
    tol = 1e-10 if prec == btam.FP64 else 1e-5
    for call in range(2):
        got = call_noalloc(gpu_tables, prec, n, inp, torch)
        scale = max(1.0, np.abs(ref["Rq"]).max())
        assert np.max(np.abs(got["V0"] - ref["V0"])) <= tol * np.abs(ref["V0"]).max(), call
        assert np.max(np.abs(got["Rq"] - ref["Rq"])) <= tol * scale, call
        assert np.max(np.abs(got["Rs"] - ref["Rs"])) <= tol * scale, call
        assert np.max(np.abs(got["Rx"] - ref["Rx"])) <= tol * max(1.0, np.abs(ref["Rx"]).max())
        assert abs(got["totals"][0] - ref["totals"][0]) <= 1e-10 * abs(ref["totals"][0])


def test_noalloc_rejects_oversized_systems(gpu_tables):
    torch = pytest.importorskip("torch")
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda").data_ptr()
    code = btam.lib().btam_mf_eval_noalloc(gpu_tables.handle, btam.FP64, 16385, *([dummy] * 12),
                                           None)
    assert code == 15  # BTAM_ERR_TOO_LARGE, before any device work
