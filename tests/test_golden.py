"""Pins the CPU oracle (and the product's host verifier) to golden vectors produced
by the reference's own CUDA kernels on a B200 (tests/golden/gen_ref_golden.py)."""
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_golden.npz"
pytestmark = pytest.mark.skipif(not GOLDEN.exists(), reason="golden fixture not generated yet")


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(GOLDEN))


@pytest.mark.parametrize("log_n", [6, 9])
def test_native_twiddles(fx, log_n):
    tw = O.native_twiddles(log_n)
    # the reference leaves the unused last line slot uninitialised; compare the n - 2 written ones
    n = 1 << log_n
    assert np.array_equal(tw["line"][: n - 2], fx[f"tw{log_n}_line"][: n - 2])
    assert np.array_equal(tw["circle"], fx[f"tw{log_n}_circle"])
    assert np.array_equal(tw["iline"][: n - 2], fx[f"tw{log_n}_iline"][: n - 2])
    assert np.array_equal(tw["icircle"], fx[f"tw{log_n}_icircle"])


def test_native_ntt(fx):
    assert np.array_equal(O.native_evaluate(fx["ntt9_in"], 9), fx["ntt9_eval"])


def test_fold_twiddles(fx):
    assert np.array_equal(O.fold_twiddles(O.HALF_COSET, 8, True), fx["foldtw_hc8"])
    assert np.array_equal(O.fold_twiddles(O.HALF_ODDS, 7, False), fx["foldtw_ho7"])


def test_batch_inverse(fx):
    assert np.array_equal(O.batch_inverse(fx["binv_in"]), fx["binv_out"])


@pytest.mark.parametrize("nc", [1, 4, 16, 20])
def test_leaves(fx, nc):
    assert np.array_equal(O.leaf_hashes_capped(fx["leaf_cols"][:nc]), fx[f"leaves_c{nc}"])


def test_soa4_tiles(fx):
    s4 = fx["soa4_in"]
    leaves = np.stack([O.blake2s_words(s4[:, i]) for i in range(s4.shape[1])])
    tiles = np.stack([O.merkle_root_hashes(leaves[i:i + 1024]) for i in range(0, s4.shape[1], 1024)])
    assert np.array_equal(tiles, fx["soa4_tiles"])


def test_fold_line(fx):
    tw = O.fold_twiddles(O.HALF_ODDS, 8, False)
    assert np.array_equal(O.fold_line(fx["fold_src"], tw, fx["fold_alpha"]), fx["fold_line"])


def test_quotient(fx):
    assert np.array_equal(O.fib_quotient(fx["quot_trace"], fx["fold_alpha"]), fx["quot_out"])


@pytest.mark.parametrize("log_n,a,b", [(4, 1, 1), (5, 2, 3), (6, 1, 1), (8, 42, 99)])
def test_proof_bytes(fx, log_n, a, b):
    ref = fx[f"proof_{log_n}_{a}_{b}"].tobytes()
    assert O.prove(a, b, log_n) == ref
    assert O.verify(ref) == (0, "")
