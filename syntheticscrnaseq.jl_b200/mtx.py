"""Reading the 10x Matrix Market files that DeviceRun.write_mtx (scrna_state_write_mtx) writes.

read_10x_mtx follows the reader of experiments/compare_real_scrnaseq.jl:69-93: skip the
comment lines, read "n_genes n_cells n_nonzero", then one "gene cell count" line (1-based) per
nonzero, giving a genes x cells matrix.
"""
from __future__ import annotations

import os

import numpy as np


def read_10x_mtx(path: str, dense: bool = True):
    """genes x cells counts of a matrix.mtx file (dense int64 array, or (rows, cols, vals, shape)
    with 0-based indices when dense is False)."""
    with open(path) as f:
        lines = f.read().splitlines()
    k = 0
    while lines[k].startswith("%"):
        k += 1
    n_genes, n_cells, nnz = (int(x) for x in lines[k].split()[:3])
    body = np.loadtxt(lines[k + 1:k + 1 + nnz], dtype=np.int64, ndmin=2) if nnz else np.zeros((0, 3), np.int64)
    if body.shape[0] != nnz:
        raise ValueError(f"{path}: header announces {nnz} entries, found {body.shape[0]}")
    rows, cols, vals = body[:, 0] - 1, body[:, 1] - 1, body[:, 2]
    if not dense:
        return rows, cols, vals, (n_genes, n_cells)
    X = np.zeros((n_genes, n_cells), dtype=np.int64)
    np.add.at(X, (rows, cols), vals)
    return X


def read_names(path: str, column: int = 1):
    """Tab-separated name column of genes.tsv (the reference reads column 2) or barcodes.tsv."""
    with open(path) as f:
        return [line.rstrip("\n").split("\t")[min(column, len(line.split("\t")) - 1)] for line in f if line.strip()]
