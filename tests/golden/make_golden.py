"""Generates the golden fixtures of tests/golden/.

    python tests/golden/make_golden.py cpu   # here: scipy / sklearn / reference condense
    python tests/golden/make_golden.py gpu   # on a GPU box: the reference library itself

cpu.npz   single-linkage trees from scipy.cluster.hierarchy.linkage (the
          reference's own test oracle) for seeded float32 inputs; condensed
          trees from the reference's cuhc_condense_tree (oracle/_ref, a CPU
          function); labels and probabilities from scikit-learn 1.9's
          tree_to_labels for the same trees.
reference_gpu.npz
          outputs of the reference library (shangar21/cuhc built from its
          sources for sm_100a, oracle/_ref/libcuhc.so) with spatial pruning
          off, so ties break by original index: single-linkage trees, HDBSCAN
          trees and core distances, RNN-Ward trees. Pins the CPU oracle and the
          library to the reference itself on machines without the reference.

Inputs are regenerated from their seeds by tests/golden/inputs.py; only the
outputs are stored.
"""

import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

from inputs import CPU_CASES, GPU_CASES, make_input  # noqa: E402


def cpu():
    from scipy.cluster.hierarchy import linkage  # noqa: PLC0415

    from oracle import oracle as O  # noqa: PLC0415

    out = {}
    for name, spec in CPU_CASES.items():
        X = make_input(spec)
        if spec["kind"] == "single":
            out[f"{name}/Z"] = linkage(X.astype(np.float64), "single")
        elif spec["kind"] == "condense":
            Z = O.hdbscan_tree(X, spec["k"])[0]
            out[f"{name}/tree"] = Z
            for mcs in spec["mcs"]:
                rows = O.reference_condense_tree(Z, mcs)
                for field, array in zip(("parent", "child", "lambda", "size"), rows):
                    out[f"{name}/mcs{mcs}/{field}"] = array
                try:
                    from sklearn.cluster._hdbscan._linkage import HIERARCHY_dtype  # noqa: PLC0415
                    from sklearn.cluster._hdbscan._tree import tree_to_labels  # noqa: PLC0415
                except ImportError:
                    continue
                tree = np.empty(len(Z), dtype=HIERARCHY_dtype)
                tree["left_node"], tree["right_node"] = Z[:, 0], Z[:, 1]
                tree["value"], tree["cluster_size"] = Z[:, 2], Z[:, 3]
                for method in ("eom", "leaf"):
                    labels, probs = tree_to_labels(tree, min_cluster_size=mcs,
                                                   cluster_selection_method=method)
                    out[f"{name}/mcs{mcs}/{method}/labels"] = labels
                    out[f"{name}/mcs{mcs}/{method}/probabilities"] = probs
    np.savez_compressed(HERE / "cpu.npz", **out)
    print(f"wrote {len(out)} arrays to cpu.npz")


def gpu():
    from oracle import oracle as O  # noqa: PLC0415

    out = {}
    for name, spec in GPU_CASES.items():
        X = make_input(spec)
        if spec["kind"] == "single":
            out[f"{name}/Z"] = O.reference_linkage(X, "single", "mst", pruning="never")
        elif spec["kind"] == "hdbscan":
            Z, core = O.reference_hdbscan_tree(X, spec["k"], pruning="never")
            out[f"{name}/Z"], out[f"{name}/core"] = Z, core
        elif spec["kind"] == "ward":
            out[f"{name}/Z"] = O.reference_linkage(X, "ward", "rnn", pruning="never")
    target = ROOT / "tests" / "golden" / "reference_gpu.npz"
    np.savez_compressed(target, **out)
    print(f"wrote {len(out)} arrays to {target}")


if __name__ == "__main__":
    {"cpu": cpu, "gpu": gpu}[sys.argv[1]]()
