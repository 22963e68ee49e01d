"""Result CSVs with the reference's file layout and columns, so its analysis scripts keep working.

results/<dataset>/<run_name>/<instance>.csv: one row per (instance, dataset, seed, run), replaced
on rerun (models/spectral_annealing.py:722-771). results/<dataset>/<run_name>/alphas/
<instance>_alphas.csv: the per-alpha rows of a sweep; a rerun of the same (instance, dataset, seed,
run) replaces all of its rows, and rows are sorted by (seed, alpha)
(models/spectral_annealing.py:773-814).
"""
from __future__ import annotations

from pathlib import Path
from typing import Dict, List

import pandas as pd


def _stem(instance_name: str) -> str:
    return instance_name.replace(".txt", "")


def store_general(dataset: str, run_name: str, instance_name: str, row: Dict) -> Path:
    out_dir = Path("results") / dataset / run_name
    out_dir.mkdir(parents=True, exist_ok=True)
    path = out_dir / f"{_stem(instance_name)}.csv"
    new = pd.DataFrame([row])
    if path.exists():
        old = pd.read_csv(path, float_precision="round_trip")
        if not old.empty:
            same = ((old["instance_name"] == row["instance_name"]) & (old["dataset"] == row["dataset"])
                    & (old["seed"] == row["seed"]) & (old["solver_name"] == row["solver_name"]))
            if same.any():
                for key, value in row.items():
                    old.loc[same, key] = value
                new = old
            else:
                new = pd.concat([old, new], ignore_index=True)
    new.to_csv(path, index=False, encoding="utf-8")
    return path


def store_alphas(dataset: str, run_name: str, instance_name: str, seed, rows: List[Dict]) -> Path:
    if not rows:
        return None
    out_dir = Path("results") / dataset / run_name / "alphas"
    out_dir.mkdir(parents=True, exist_ok=True)
    path = out_dir / f"{_stem(instance_name)}_alphas.csv"
    new = pd.DataFrame(rows)
    if path.exists():
        old = pd.read_csv(path, float_precision="round_trip")
        same = ((old["instance_name"] == instance_name) & (old["dataset"] == dataset)
                & (old["seed"].isna() if seed is None else old["seed"] == seed)
                & (old["solver_name"] == run_name))
        new = pd.concat([old[~same], new], ignore_index=True)
    new = new.sort_values(["seed", "alpha"]).reset_index(drop=True)
    new.to_csv(path, index=False, encoding="utf-8")
    return path
