"""CPU checks of the C-ABI library: it loads without a GPU, exports every symbol
include/vstark.h declares, and its host-side verifier accepts oracle proofs and
rejects tampered ones (no device calls)."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
import vortexstark_b200 as V


def test_header_parses_all_entry_points():
    fns = V.declared_functions()
    # the reference's commitment-path FFI (src/cuda/ffi.rs) plus the vs_* API
    for name in ["cuda_circle_ntt_evaluate", "cuda_circle_ntt_interpolate", "cuda_circle_ntt_evaluate_batch",
                 "cuda_circle_ntt_interpolate_batch", "cuda_circle_ntt_layer", "cuda_bit_reverse_m31",
                 "cuda_eval_at_point", "cuda_stwo_ntt_evaluate", "cuda_stwo_ntt_interpolate",
                 "cuda_compute_fold_twiddle_sources", "cuda_compute_fold_twiddle_sources_stream",
                 "cuda_batch_inverse_m31", "cuda_batch_inverse_m31_stream", "cuda_compute_coset_points",
                 "cuda_squash_x", "cuda_extract_and_squash", "cuda_fibonacci_quotient", "cuda_zero_pad",
                 "cuda_fibonacci_quotient_chunk", "cuda_fibonacci_quotient_chunk_stream", "cuda_interleave_u32",
                 "cuda_fold_line_soa", "cuda_fold_circle_into_line_soa", "cuda_merkle_hash_leaves",
                 "cuda_merkle_hash_nodes", "cuda_merkle_reduce_to_root", "cuda_merkle_commit_small_soa4",
                 "cuda_merkle_hash_leaves_merge_soa4", "cuda_merkle_tiled_soa4", "cuda_merkle_tiled_soa4_stream",
                 "cuda_merkle_tiled_generic", "cuda_build_leaves_lifted", "cuda_accumulate_numerators",
                 "cuda_compute_quotients_combine", "cuda_bit_reverse_qm31", "cuda_device_sync",
                 "vs_prove_fib", "vs_verify_fib", "vs_commit_columns", "vs_fri_fold_commit", "vs_lde_stwo"]:
        assert name in fns, name


def test_library_exports_every_declared_symbol():
    raw = C.CDLL(str(V.LIB_PATH))
    missing = [n for n in V.declared_functions() if not hasattr(raw, n)]
    assert not missing, missing
    assert V.lib().vs_version().startswith(b"vstark-b200")


def _verify(proof: bytes):
    buf = (C.c_uint8 * len(proof)).from_buffer_copy(proof)
    err = C.create_string_buffer(256)
    rc = V.lib().vs_verify_fib(buf, len(proof), err, 256)
    return rc, err.value.decode()


@pytest.mark.parametrize("log_n,a,b", [(4, 1, 1), (6, 2, 3), (8, 42, 99)])
def test_product_verifier_accepts_oracle_proofs(log_n, a, b):
    assert _verify(O.prove(a, b, log_n)) == (0, "")


def test_product_verifier_rejects_tampering():
    proof = bytearray(O.prove(1, 1, 6))
    for word in (5, 13, 22):  # trace root, quotient root, first FRI root
        t = bytearray(proof)
        t[4 * word] ^= 1
        rc, msg = _verify(bytes(t))
        assert rc != 0 and msg
    assert _verify(bytes(proof[:-4]))[0] != 0
