"""Writes large_proofs.json: SHA-256 digests of the oracle's Fibonacci proofs at
full sizes (log_n 24 and 28, a0 = 1, a1 = the first seeded uniform M31 of
SplitMix64 seed 0x56530002, and a0 = a1 = 1), so GPU tests can check full-size
proofs byte for byte without minutes of CPU work at test time.

    python tests/golden/gen_large_digests.py [log_n ...]

The oracle is pinned to the reference's own kernels at small sizes (ref_golden.npz);
at log_n = 28 it needs ~40 GB of host memory and several minutes on 8 threads."""
import hashlib
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))
import oracle_lib as O  # noqa: E402
from vortexstark_b200.workloads import SplitMix64  # noqa: E402

OUT = HERE / "large_proofs.json"


def main(sizes):
    data = json.loads(OUT.read_text()) if OUT.exists() else {}
    a1 = SplitMix64(0x56530002).m31()
    for log_n in sizes:
        for a, b in ((1, a1), (1, 1)):
            t0 = time.time()
            proof = O.prove(a, b, log_n)
            rc, err = O.verify(proof)
            assert rc == 0, err
            data[f"{log_n}:{a}:{b}"] = {"log_n": log_n, "a": a, "b": b, "len": len(proof),
                                        "sha256": hashlib.sha256(proof).hexdigest()}
            print(log_n, a, b, len(proof), f"{time.time() - t0:.1f}s", flush=True)
            OUT.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main([int(x) for x in sys.argv[1:]] or [24, 28])
