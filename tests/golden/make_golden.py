"""Generate the golden vectors in this directory from the reference's own Python TR-SVD.

Runs ``trdecomposition/high_order_GPUs/python_GPUs/T3F.py`` (functions ``genTRTensor``,
``TRdecomposition`` and ``reCover``, lines 9-79) unmodified, with a small NumPy stand-in
for the TensorFlow calls it makes (reshape/transpose in C order, matmul, linalg.svd
returning (s, u, v), linalg.diag, linalg.norm, constant).  TensorFlow itself is not
installed here; every TensorFlow call the file makes has an exact NumPy equivalent.

With r0 = r_d = 1 the same function is a TT-SVD, which pins the TT chain as well.

Usage (only where the reference checkout exists):
    python tests/golden/make_golden.py /root/reference
Writes ``tr6_python_ref.npz``, ``tr6_python_ref_noisy.npz`` and ``tt6_python_ref.npz``.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types
import unittest

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _tf_stub(svd_log: list):
    tf = types.ModuleType("tensorflow")
    tf.float32 = types.SimpleNamespace(as_numpy_dtype=np.float32)
    tf.float64 = types.SimpleNamespace(as_numpy_dtype=np.float64)
    tf.reshape = lambda x, shape: np.reshape(np.asarray(x), shape)
    tf.transpose = lambda x, perm: np.transpose(np.asarray(x), perm)
    tf.matmul = lambda a, b: np.matmul(np.asarray(a), np.asarray(b))
    tf.constant = lambda x: np.asarray(x)

    def svd(x, full_matrices=False):
        u, s, vh = np.linalg.svd(np.asarray(x), full_matrices=full_matrices)
        svd_log.append(s.copy())
        return s, u, vh.T

    tf.linalg = types.SimpleNamespace(
        svd=svd,
        diag=lambda s: np.diag(np.asarray(s)),
        norm=lambda x: np.linalg.norm(np.asarray(x).ravel()),
    )
    tf.compat = types.SimpleNamespace(v1=types.SimpleNamespace(enable_eager_execution=lambda: None))
    tf.test = types.SimpleNamespace(TestCase=unittest.TestCase, main=lambda: None)
    return tf


def load_reference(ref_root: str, svd_log: list):
    sys.modules["tensorflow"] = _tf_stub(svd_log)
    path = os.path.join(ref_root, "trdecomposition", "high_order_GPUs", "python_GPUs", "T3F.py")
    spec = importlib.util.spec_from_file_location("ref_t3f_tr6", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def run_case(mod, svd_log, k, i, noise=0.0, seed=7):
    G = [0] * 7
    x = np.asarray(mod.genTRTensor(G, k, i, np.float64), dtype=np.float64)
    if noise:
        rng = np.random.default_rng(seed)
        x = x + noise * np.linalg.norm(x) / np.sqrt(x.size) * rng.standard_normal(x.shape)
    svd_log.clear()
    G = [0] * 7
    mod.TRdecomposition(x, G, k, i)
    cores = [np.array(G[j], dtype=np.float64) for j in range(1, 7)]
    sig = [s.copy() for s in svd_log]
    rec = np.asarray(mod.reCover(list(G), k, i))
    err = float(np.linalg.norm((x - rec).ravel()) / np.linalg.norm(x.ravel()))
    out = {"x": x, "k": np.array(k), "i": np.array(i), "err": np.array(err)}
    for j, c in enumerate(cores):
        out[f"core{j + 1}"] = c
    for j, s in enumerate(sig):
        out[f"sigma{j + 1}"] = s
    return out


def main(ref_root: str):
    svd_log: list = []
    mod = load_reference(ref_root, svd_log)
    cases = {
        "tr6_python_ref.npz": dict(k=[2, 2, 3, 3, 3, 3, 2], i=6),
        "tr6_python_ref_noisy.npz": dict(k=[2, 2, 3, 3, 3, 3, 2], i=6, noise=1e-3),
        "tt6_python_ref.npz": dict(k=[1, 3, 4, 4, 3, 2, 1], i=5, noise=1e-4),
    }
    for name, kw in cases.items():
        out = run_case(mod, svd_log, **kw)
        np.savez_compressed(os.path.join(HERE, name), **out)
        print(name, "err", float(out["err"]))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
