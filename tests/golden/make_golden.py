"""Generate the golden fixtures in tests/golden/ by running the REFERENCE solver code.

    python tests/golden/make_golden.py [--reference /path/to/reference]

The reference (Vgueca/SpecAnn) is CuPy-only and CuPy is not installed here, so the script installs
the NumPy/SciPy stand-in of tests/golden/_cupy_shim.py under the names cupy/cupyx and then imports
the reference's own models/spectral_annealing.py, models/spec_adj.py and models/spec_signed_lap.py
unchanged. Each case loads an instance with the reference's utils/data_loader.py, runs the
reference solver's solve(J) in a scratch directory, and freezes what it produced:

  * the per-alpha CSV rows the reference writes (alpha, lambda1, pred_residual, pred_accepted,
    eigsh_retry, raw_energy, energy, candidate, local_search_iterations, ...);
  * for every alpha, the rounding vector x = D^{-1/2} y and the eigenvector y it rounded (captured
    around _solve_eigenvalue_problem_pred) and the rounded spins (captured around
    _compute_spin_signature);
  * the returned best energy and best spins; the normalisation factor.

The fixtures are .npz files named after the case. The script needs the reference tree; the tests
only need the committed .npz files.
"""
import argparse
import contextlib
import io
import json
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

CASES = [
    # name, dataset, instance, solver module/class, params
    ("tiny_ba20_specann32", "barabasi_albert_3ins_m10_tiny", "ba_20_1_0.txt", "spectral_annealing", {}),
    ("tiny_ba100_specann32", "barabasi_albert_3ins_m10_tiny", "ba_100_1_0.txt", "spectral_annealing", {}),
    ("tiny_ba190_specann64", "barabasi_albert_3ins_m10_tiny", "ba_190_1_2.txt", "spectral_annealing",
     {"precision": 64}),
    ("ba128_secant32", "barabasi_albert_10ins_m20", "ba_128_1_0.txt", "spectral_annealing",
     {"pred_mode": "secant", "num_alphas": 32}),
    ("er128_prev_linear32", "erdos_renyi_10ins_m20", "er_128_1_0.txt", "spectral_annealing",
     {"pred_mode": "prev", "schedule": "linear", "num_alphas": 24}),
    ("er1024_linear16_nols32", "erdos_renyi_10ins_m20", "er_1024_1_0.txt", "spectral_annealing",
     {"schedule": "linear", "num_alphas": 16, "use_local_search": False}),
    ("tiny_ba100_specadj32", "barabasi_albert_3ins_m10_tiny", "ba_100_1_0.txt", "spec_adj", {}),
    ("tiny_ba120_specsignedlap32", "barabasi_albert_3ins_m10_tiny", "ba_120_1_0.txt", "spec_signed_lap", {}),
]

CLASSES = {"spectral_annealing": "SpectralAnnealing", "spec_adj": "Alpha0GPU",
           "spec_signed_lap": "Alpha1GPU"}


def run_case(ref: Path, name, dataset, instance, module, params, seed=42):
    import importlib
    import pandas as pd
    from utils.data_loader import DataLoader

    loader = DataLoader(dataset, datasets_path=str(ref / "datasets"))
    J = loader.load_instance(instance)
    mod = importlib.import_module(f"models.{module}")
    cls = getattr(mod, CLASSES[module])
    captured = {"x": [], "y": [], "spins": [], "alpha": []}

    if module == "spectral_annealing":
        orig_solve = cls._solve_eigenvalue_problem_pred
        orig_sig = cls._compute_spin_signature

        def solve_pred(self, *a, **k):
            out = orig_solve(self, *a, **k)
            captured["alpha"].append(a[3])
            captured["x"].append(np.array(out[1][:, 0]))
            captured["y"].append(np.array(out[2][:, 0]))
            return out

        def sig(self, spins):
            captured["spins"].append(np.array(spins))
            return orig_sig(self, spins)

        cls._solve_eigenvalue_problem_pred = solve_pred
        cls._compute_spin_signature = sig
    with tempfile.TemporaryDirectory() as tmp:
        cwd = os.getcwd()
        os.chdir(tmp)
        try:
            solver = cls(instance_name=instance, dataset=dataset, run_name=name, random_seed=seed, **params)
            with contextlib.redirect_stdout(io.StringIO()):
                energy, spins, _ = solver.solve(J)
            alphas_csv = Path(tmp) / "results" / dataset / name / "alphas" / (instance.replace(".txt", "") + "_alphas.csv")
            general_csv = Path(tmp) / "results" / dataset / name / (instance.replace(".txt", "") + ".csv")
            rows = pd.read_csv(alphas_csv) if alphas_csv.exists() else None
            general = pd.read_csv(general_csv)
        finally:
            os.chdir(cwd)
            if module == "spectral_annealing":
                cls._solve_eigenvalue_problem_pred = orig_solve
                cls._compute_spin_signature = orig_sig
    out = dict(indptr=J.indptr.astype(np.int64), indices=J.indices.astype(np.int32),
               data=J.data.astype(np.float64), n=np.int64(J.shape[0]),
               best_energy=np.float64(energy), best_spins=np.asarray(spins).astype(np.int8),
               normalization=np.float64(getattr(solver, "_normalization_factor", np.nan)),
               params=json.dumps(dict(params, seed=seed, module=module)))
    if rows is not None:
        for col in ("alpha", "lambda1", "pred_residual", "raw_energy", "energy", "degree_scale",
                    "energy_bound"):
            out[f"row_{col}"] = rows[col].to_numpy(dtype=np.float64)
        out["row_pred_accepted"] = rows["pred_accepted"].map(
            lambda v: -1 if (isinstance(v, float) and np.isnan(v)) else int(bool(v))).to_numpy(np.int64)
        out["row_eigsh_retry"] = rows["eigsh_retry"].astype(bool).to_numpy()
        out["row_candidate"] = rows["candidate"].fillna(-1).to_numpy(np.int64)
        out["row_ls_iterations"] = rows["local_search_iterations"].to_numpy(np.int64)
    out["general_local_search_iterations"] = np.int64(general["local_search_iterations"].iloc[0])
    if captured["x"]:
        out["cap_alpha"] = np.asarray(captured["alpha"], dtype=np.float64)
        out["cap_x"] = np.stack(captured["x"])
        out["cap_y"] = np.stack(captured["y"])
        if captured["spins"]:
            out["cap_spins"] = np.stack(captured["spins"]).astype(np.int8)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    ref = Path(args.reference)
    import _cupy_shim
    _cupy_shim.install()
    sys.path.insert(0, str(ref))
    for name, dataset, instance, module, params in CASES:
        if args.only and args.only != name:
            continue
        out = run_case(ref, name, dataset, instance, module, params)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"{name}: n={int(out['n'])} best_energy={float(out['best_energy'])}")


if __name__ == "__main__":
    main()
