"""GPU: full-size Fibonacci proofs (log_n 24 and 28) byte for byte against the
oracle, through SHA-256 digests of the oracle's proofs (tests/golden/large_proofs.json,
written by tests/golden/gen_large_digests.py: at log_n = 28 the oracle needs
minutes of CPU time and ~40 GB of host memory, too much to rerun per test).

Both the drop-in vs_prove_fib path and the graph-captured prover are checked,
and every proof must verify."""
import hashlib
import json
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from vortexstark_b200 import api  # noqa: E402

DIGESTS = Path(__file__).resolve().parent / "golden" / "large_proofs.json"
CASES = json.loads(DIGESTS.read_text()) if DIGESTS.exists() else {}


@pytest.mark.parametrize("key", sorted(CASES, key=lambda k: [int(x) for x in k.split(":")]))
def test_full_size_proof_matches_oracle_digest(key):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = CASES[key]
    plain = api.prove_fib(c["a"], c["b"], c["log_n"])
    with api.Engine(1) as eng:
        graph = eng.wait(eng.submit(api.fib_job(c["log_n"], c["a"], c["b"])))[0]
    assert graph == plain
    assert len(plain) == c["len"]
    assert hashlib.sha256(plain).hexdigest() == c["sha256"]
    assert api.verify_fib(plain) == (True, "")


@pytest.mark.parametrize("split", [3, 5])
@pytest.mark.parametrize("key", sorted(CASES, key=lambda k: [int(x) for x in k.split(":")]))
def test_full_size_proof_with_merkle_split(key, split):
    """The prover's trees of 2^20+ leaves reach their tile roots through 2^split
    subtree roots per tile; the proof bytes must not change."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = CASES[key]
    api.set_merkle_split(split)
    try:
        plain = api.prove_fib(c["a"], c["b"], c["log_n"])
        with api.Engine(1) as eng:
            graph = eng.wait(eng.submit(api.fib_job(c["log_n"], c["a"], c["b"])))[0]
    finally:
        api.set_merkle_split(0)
    assert graph == plain
    assert hashlib.sha256(plain).hexdigest() == c["sha256"]
