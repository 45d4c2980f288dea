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


def device_outputs(n, torch):
    """Caller-owned device buffers for the outputs."""
    return dict(V0=torch.zeros(n, dtype=torch.float64, device="cuda"),
                Rq=torch.zeros((n, 3), dtype=torch.float64, device="cuda"),
                Rs=torch.zeros(n, dtype=torch.float64, device="cuda"),
                Rx=torch.zeros(n, dtype=torch.float64, device="cuda"),
                totals=torch.zeros(4, dtype=torch.float64, device="cuda"))


def call_noalloc(tables, prec, n, inp, torch, out=None):
    if out is None:
        out = device_outputs(n, torch)
    p = lambda t: t.data_ptr()
    code = btam.lib().btam_mf_eval_noalloc(
        tables.handle, prec, n, p(inp["pos4"]), p(inp["xb"]), p(inp["code"]),
        p(inp["owner"]), p(inp["gamma"]), p(inp["offs"]), p(inp["idx"]), p(out["V0"]),
        p(out["Rq"]), p(out["Rs"]), p(out["Rx"]), p(out["totals"]),
        torch.cuda.current_stream().cuda_stream)
    assert code == 0, btam.STATUS.get(code, code)
    return {k: v.cpu().numpy() for k, v in out.items()}


def near_limit_system():
    """A periodic hcp Mg-H block of 14 x 15 x 13 hexagonal cells with H on
    every tetrahedral site: 16380 sites, just under the entry point's
    16384-site limit, so the top of the fixed scratch array is used."""
    return lattice.supercell(14, 15, 13, h_fraction=1.0, x_range=(0.0, 0.3),
                             sigma_range=(0.08, 0.15), jitter=0.02, T=400.0, seed=11)


def check_against(got, ref, prec, call):
    # tolerances of the parity tests: FP64 1e-10 relative, FP32C 1e-6 relative
    # energy and 1e-5 on residual components
    tol = 1e-10 if prec == btam.FP64 else 1e-5
    tol_e = 1e-10 if prec == btam.FP64 else 1e-6
    scale = max(1.0, np.abs(ref["Rq"]).max())
    assert np.max(np.abs(got["V0"] - ref["V0"])) <= tol * np.abs(ref["V0"]).max(), call
    assert np.max(np.abs(got["Rq"] - ref["Rq"])) <= tol * scale, call
    assert np.max(np.abs(got["Rs"] - ref["Rs"])) <= tol * scale, call
    assert np.max(np.abs(got["Rx"] - ref["Rx"])) <= tol * max(1.0, np.abs(ref["Rx"]).max())
    assert abs(got["totals"][0] - ref["totals"][0]) <= tol_e * abs(ref["totals"][0]), call


@pytest.mark.parametrize("size", ["small", "near_limit"])
@pytest.mark.parametrize("prec", [btam.FP64, btam.FP32C])
def test_noalloc_matches_allocating_entry_point(gpu_tables, prec, size):
    torch = pytest.importorskip("torch")
    s = lattice.config1(seed=7) if size == "small" else near_limit_system()
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    ref = S.evaluate(prec)
    n = len(s["x"])
    assert size == "small" or 16000 < n <= 16384
    inp = device_inputs(S, s, torch)
    for call in range(2):
        check_against(call_noalloc(gpu_tables, prec, n, inp, torch), ref, prec, call)
    S.close()


def test_noalloc_allocates_nothing(gpu_tables):
    """The defining property: with inputs and outputs in place, calls change
    neither the library's device pool nor the device's free memory."""
    torch = pytest.importorskip("torch")
    s = lattice.config1(seed=7)
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    n = len(s["x"])
    inp = device_inputs(S, s, torch)
    out = device_outputs(n, torch)
    # one call per form first: they load the kernels' code and look the
    # scratch up
    for prec in (btam.FP64, btam.FP32C):
        call_noalloc(gpu_tables, prec, n, inp, torch, out)
    torch.cuda.synchronize()
    pool0, free0 = btam.pool_usage(), torch.cuda.mem_get_info()[0]
    for prec in (btam.FP64, btam.FP32C, btam.FP64):
        call_noalloc(gpu_tables, prec, n, inp, torch, out)
    torch.cuda.synchronize()
    assert btam.pool_usage() == pool0
    assert torch.cuda.mem_get_info()[0] == free0
    S.close()


def test_noalloc_rejects_oversized_systems(gpu_tables):
    torch = pytest.importorskip("torch")
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda").data_ptr()
    code = btam.lib().btam_mf_eval_noalloc(gpu_tables.handle, btam.FP64, 16385, *([dummy] * 12),
                                           None)
    assert code == 15  # BTAM_ERR_TOO_LARGE, before any device work
