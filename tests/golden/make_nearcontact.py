"""Generate tests/golden/nearcontact_pairs.npz: near-contact training pairs
made by the method itself on the GPU (FP64 path, frozen two-sphere runs on a
64^3 coarse grid with a = 5 and a 128^3 fine grid with a = 10, dynamically
similar units; kapsel_old_b200.nearcontact.generate).

    python tests/golden/make_nearcontact.py [--n 2048] [--seed 5]

Needs a B200 (the pairs are GPU runs, not oracle runs; the FP64 GPU step is
pinned to the oracle by the parity tests)."""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from kapsel_old_b200 import nearcontact as nc  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--steps", type=int, default=nc.N_STEPS)
    ap.add_argument("--out", default=os.path.join(HERE, "nearcontact_pairs.npz"))
    a = ap.parse_args()
    t0 = time.time()
    d = nc.generate(a.n, a.seed, a.steps, progress=256)
    d["seed"] = a.seed
    np.savez_compressed(a.out, **{k: np.asarray(v) for k, v in d.items()})
    print(f"{a.n} pairs in {time.time() - t0:.1f} s -> {a.out}")


if __name__ == "__main__":
    main()
