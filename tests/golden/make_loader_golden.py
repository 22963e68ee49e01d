"""Golden outputs of the reference's instance loader (utils/data_loader.py), for the native loader
test (tests/test_loader.py).

    python tests/golden/make_loader_golden.py [--reference /path/to/reference]

`write_instance_files` writes small synthetic instance files in the two formats the loader reads,
with the irregular lines the loader must handle (comments, blank lines, short and unparsable
lines, float-formatted node numbers, self-loops, out-of-range nodes, duplicate edges, zero and
nonzero fields, isolated nodes). The script loads them with the reference's DataLoader and freezes
the CSR arrays and index fields in loader_golden.npz. The test needs only the .npz.
"""
import argparse
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def write_instance_files(root: Path):
    """Files as (dataset folder, file name) under root; deterministic."""
    rng = np.random.default_rng(20251203)
    out = []
    # linear-bias format, nonzero fields (bias node), one isolated node (7), duplicates
    d = root / "synthetic_lb"
    d.mkdir(parents=True, exist_ok=True)
    n = 12
    lines = [f"{n} 0"]
    h = [0.0] * n
    h[2], h[5], h[9] = 3.0, -1.5, 2.0
    lines += [repr(x) for x in h]
    edges = []
    for _ in range(30):
        i, j = rng.integers(1, n + 1, 2)
        if 7 in (i, j):
            continue
        edges.append(f"{i} {j} {int(rng.integers(-5, 6))}")
    edges += ["# a comment", "", "% another", "3", "4 5", "x y 1", "3.0 4.0 2.5", "1 1 9", "0 3 1",
              f"{n + 1} 2 1", "2 3 1 extra", "2 3 -1", "6 8 nan-ish"]
    lines += edges
    (d / "lb_12.txt").write_text("\n".join(lines) + "\n")
    out.append(("synthetic_lb", "lb_12.txt"))
    # linear-bias format, all fields zero (no bias node)
    n = 9
    lines = [f"{n} 0"] + ["0"] * n
    for _ in range(25):
        i, j = rng.integers(1, n + 1, 2)
        lines.append(f"{i} {j} {float(rng.normal()):.6f}")
    (d / "lb_9_nofield.txt").write_text("\n".join(lines) + "\n")
    out.append(("synthetic_lb", "lb_9_nofield.txt"))
    # Gset format: weights negated, isolated node 4, duplicates that cancel
    d = root / "synthetic_Gset"
    d.mkdir(parents=True, exist_ok=True)
    n = 10
    lines = [f"{n} 0"]
    for _ in range(28):
        i, j = rng.integers(1, n + 1, 2)
        if 4 in (i, j):
            continue
        lines.append(f"{i} {j} {int(rng.integers(1, 4))}")
    lines += ["1 2 1", "2 1 -1", "# c", "5 5 3", "11 1 1"]
    (d / "g_10.txt").write_text("\n".join(lines) + "\n")
    out.append(("synthetic_Gset", "g_10.txt"))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    import warnings
    from utils.data_loader import DataLoader
    res = {}
    with tempfile.TemporaryDirectory() as tmp:
        files = write_instance_files(Path(tmp))
        for k, (ds, name) in enumerate(files):
            with warnings.catch_warnings():
                warnings.simplefilter("ignore")
                J, idx = DataLoader(ds, datasets_path=tmp).load_instance(name, return_index=True)
            J = J.tocsr()
            res[f"f{k}_indptr"] = J.indptr.astype(np.int64)
            res[f"f{k}_indices"] = J.indices.astype(np.int32)
            res[f"f{k}_data"] = J.data.astype(np.float64)
            res[f"f{k}_shape"] = np.array(J.shape, dtype=np.int64)
            res[f"f{k}_node_ids"] = np.asarray(idx.node_ids, dtype=np.int64)
            res[f"f{k}_meta"] = np.array([idx.n_original, idx.n_solve, idx.bias_node_index,
                                          int(idx.weights_negated)], dtype=np.int64)
            res[f"f{k}_J_sum"] = np.float64(idx.J_sum)
    np.savez_compressed(HERE / "loader_golden.npz", **res)
    print(f"{len(files)} files -> loader_golden.npz")


if __name__ == "__main__":
    main()
