"""The per-term plugin table on the device against the reference's own
functions.

tests/golden/termfns.npz holds, for every slot of potential_function
(Macros.hpp:252-278) of rho_ij, V_pair_ij, V_dipole_ij1j2 and
V_quadrupole_ij1j2 (MgHx-ADP.cpp:526-2434) and every direction, the
reference's output at seeded geometries (tests/golden/make_golden.py,
--termfns).  tests/golden/terms.npz holds the reference's degree-3
averages of the same terms (Quadrature-Hermitian-3th.cpp:36-378).

Tolerances, relative to max(1, |golden|) per slot: F, dF_dq, dF_dn and the
finite-difference gradient 1e-12 (the same operations in the same order;
the FD gradient divides differences of values that agree to rounding by
12e-4, so 1e-12 holds with room); the analytic Hessian blocks 1e-10 (formed
from the terms' radial, vector and tensor parts in another order than the
reference's); the FD Hessian 1e-4 absolute on entries of order 1 (second
differences with step 1e-4 amplify the rounding of F by 1e8 / 12);
quadratures 1e-12."""
import os

import numpy as np
import pytest

import btam

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = {0: 1e-12, 1: 1e-12, 2: 1e-10, 3: 1e-12, 5: 1e-12}


def rows():
    d = dict(np.load(os.path.join(GOLD, "termfns.npz")))
    keys = sorted({tuple(m[:3]) for m in d["meta"]})
    return d, keys


def test_every_slot_of_every_term(gpu_tables):
    d, keys = rows()
    for term, fn, direction in keys:
        sel = np.all(d["meta"][:, :3] == (term, fn, direction), axis=1)
        out = gpu_tables.term(term, fn, direction, d["q"][sel], d["x"][sel], d["species"][sel])
        gold = d["out"][sel]
        err = np.abs(out - gold)
        if fn == 4:
            # the FD Hessian: diagonal entries only, the rest 0 on both sides
            assert np.all(out[:, [1, 2, 3, 5, 6, 7]] == 0.0)
            assert err.max() <= 1e-4 * max(1.0, np.abs(gold).max()), (term, fn, direction)
        else:
            assert err.max() <= TOL[fn] * max(1.0, np.abs(gold).max()), (term, fn, direction,
                                                                         err.max())


def test_gradient_slots_agree_with_the_hessian_slots(gpu_tables):
    """Internal consistency at the same geometries: dF_dq matches dF_dq_FD
    up to the finite differences' truncation and the reference's stale
    coordinate (the second and third components are taken with the earlier
    coordinates left 2 dr away: an error of order 2e-4 |H|), and the
    analytic Hessian's diagonal blocks match the FD Hessian's diagonal."""
    d, _ = rows()
    for term in range(4):
        ns = 2 if term < 2 else 3
        sel = np.all(d["meta"][:, :2] == (term, 0), axis=1)
        q, x, sp = d["q"][sel], d["x"][sel], d["species"][sel]
        for s in range(ns):
            g = gpu_tables.term(term, 1, s, q, x, sp)[:, :3]
            gf = gpu_tables.term(term, 3, s, q, x, sp)[:, :3]
            assert np.abs(g - gf).max() <= 1e-3 * max(1.0, np.abs(g).max())
            blk = s * (ns + 1)
            h = gpu_tables.term(term, 2, blk, q, x, sp)[:, [0, 4, 8]]
            hf = gpu_tables.term(term, 4, blk, q, x, sp)[:, [0, 4, 8]]
            assert np.abs(h - hf).max() <= 1e-4 * max(1.0, np.abs(h).max())


def test_degree3_quadratures(gpu_tables):
    d = dict(np.load(os.path.join(GOLD, "terms.npz")))
    meta = d["meta"]
    for key in sorted({tuple(m) for m in meta}):
        term, mode, slot, ns, coinc = key
        sel = np.all(meta == key, axis=1)
        q = d["q"][sel]
        out = gpu_tables.term_quadrature(term, mode, slot, q, d["sigma"][sel], d["x"][sel],
                                         d["species"][sel], coincident=coinc)
        k = 3 if mode == 1 else 1
        gold = d["out"][sel][:, :k]
        assert np.abs(out[:, :k] - gold).max() <= 1e-12 * max(1.0, np.abs(gold).max()), key
        assert np.all(out[:, k:] == 0.0)


def test_arguments_are_checked(gpu_tables):
    q = np.zeros((1, 9))
    q[0, 3] = 2.5
    x = np.ones((1, 3))
    sp = np.full((1, 3), 12)
    with pytest.raises(btam.BtamError):
        gpu_tables.term(4, 0, 0, q, x, sp)          # no fifth term
    with pytest.raises(btam.BtamError):
        gpu_tables.term(0, 1, 2, q, x, sp)          # pair terms have 2 sites
    with pytest.raises(btam.BtamError):
        gpu_tables.term(2, 2, 9, q, x, sp)          # 3 x 3 blocks
    with pytest.raises(btam.BtamError):
        gpu_tables.term(0, 0, 0, q, x, np.full((1, 3), 8))   # oxygen
    with pytest.raises(btam.BtamError):
        gpu_tables.term_quadrature(1, 0, 0, q, np.full((1, 3), 0.1), x, sp, coincident=True)
    assert gpu_tables.term(0, 0, 0, q[:0], x[:0], sp[:0]).shape == (0, 9)


def test_reference_style_caller_of_the_term_table(tmp_path):
    """A caller of the reference's term constructors (potential_function
    function pointers, one geometry per call) built against the drop-ins of
    include/btam_dmd_equations.hpp gets the reference's values."""
    import struct
    import subprocess
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    import compat_build
    d, _ = rows()
    rng = np.random.default_rng(5)
    pick = np.sort(rng.choice(len(d["meta"]), 240, replace=False))
    inp, out = tmp_path / "terms.bin", tmp_path / "terms.out"
    with open(inp, "wb") as f:
        f.write(struct.pack("i", len(pick)))
        for r in pick:
            f.write(np.asarray(d["meta"][r, :3], np.int32).tobytes())
            f.write(d["q"][r].astype(np.float64).tobytes())
            f.write(d["x"][r].astype(np.float64).tobytes())
            f.write(np.asarray(d["species"][r], np.int32).tobytes())
    probe = compat_build.build_probe()
    res = subprocess.run([probe, btam.TABLES_DIR, str(inp), str(out), "terms"],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    raw = open(out, "rb").read()
    vals = np.frombuffer(raw[:-4], np.float64).reshape(len(pick), 9)
    assert struct.unpack("i", raw[-4:])[0] == 0
    for k, r in enumerate(pick):
        fn = d["meta"][r, 1]
        tol = 1e-4 if fn == 4 else TOL[fn]
        gold = d["out"][r]
        assert np.abs(vals[k] - gold).max() <= tol * max(1.0, np.abs(gold).max()), r


def test_fifth_degree_rule(gpu_tables):
    """The reference's 5th-degree rule over the pair measure
    (Quadrature-Hermitian-5th.cpp:31-432) on the device against the
    reference build's values (tests/golden/quad5.npz): averages of F and
    dF_dq within 1e-12, of d2F_dq2 within 1e-10 (the analytic blocks'
    tolerance)."""
    d = dict(np.load(os.path.join(GOLD, "quad5.npz")))
    for key in sorted({tuple(m) for m in d["meta"]}):
        term, mode, direction = key
        sel = np.all(d["meta"] == key, axis=1)
        out = gpu_tables.term_quadrature5(term, mode, direction, d["q"][sel], d["sigma"][sel],
                                          d["x"][sel], d["species"][sel])
        gold = d["out"][sel]
        tol = 1e-10 if mode == 2 else 1e-12
        assert np.abs(out - gold).max() <= tol * max(1.0, np.abs(gold).max()), key
    with pytest.raises(btam.BtamError):
        gpu_tables.term_quadrature5(2, 0, 0, d["q"][:1], d["sigma"][:1], d["x"][:1],
                                    d["species"][:1])  # pair terms only
