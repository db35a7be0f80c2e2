"""Golden vectors from the reference itself: run the reference's CUDA
extension (rebuilt for sm_100a by ``make -C oracle ref``) on a B200 and
write energies and gradients of seeded cases to ref_golden.json.

Run on a GPU host from the repository root:
    python tests/golden/make_ref_golden.py [out.json]
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
from tests.refmod import load_reference_module  # noqa: E402

# (n, L, h, seed): params uniform in [0, 2pi) from default_rng(seed)
CASES = [
    (2, 1, 0.7, 1), (2, 3, 1.0, 2), (3, 2, 1.1, 3), (4, 2, 1.0, 4), (5, 3, 0.3, 5),
    (6, 2, 1.1, 6), (7, 4, 0.9, 7), (8, 3, 1.0, 8), (9, 2, 2.0, 9), (10, 3, 0.5, 10),
    (11, 2, 1.3, 11), (12, 3, 1.0, 12), (13, 2, 0.8, 13), (14, 2, 1.0, 14), (16, 2, 1.2, 16),
    (18, 2, 1.0, 18), (20, 2, 1.0, 20), (20, 4, 1.0, 7),
]


def params_for(n: int, L: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(0.0, 2.0 * np.pi, 2 * n * L)


def main() -> None:
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).with_name("ref_golden.json")
    ref = load_reference_module()
    if ref is None:
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    rows = []
    for n, L, h, seed in CASES:
        p = params_for(n, L, seed)
        b = ref.RingIsingCudaBackend(n, L, h, "structured_adjoint", 8, False)
        r = b.energy_and_grad(p, True, False)
        rows.append({"n": n, "L": L, "h": h, "seed": seed, "energy": float(r["energy"]),
                     "gradient": [float(x) for x in np.asarray(r["gradient"])]})
        print(n, L, h, r["energy"], flush=True)
    out.write_text(json.dumps({
        "source": "reference cpp/ rebuilt for sm_100a (oracle/_ref), strategy structured_adjoint, width 8",
        "params": "numpy default_rng(seed).uniform(0, 2pi, 2 n L)",
        "cases": rows,
    }) + "\n")
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
