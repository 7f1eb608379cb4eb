"""cuhc_b200: exact hierarchical clustering and HDBSCAN on B200 GPUs.

A drop-in for the Python API of cuhc (scipy / scikit-learn semantics):
`linkage`, `fcluster`, `AgglomerativeClustering`, `HDBSCAN` and
`pairwise_distances`, over the C ABI of libcuhc.so (include/cuhc.h).
"""

from ._batch import batched_trees
from ._distances import METRIC_IDS, pairwise_distances
from ._linkage import LINKAGE_IDS, fcluster, linkage
from ._radius import load_radius_model, radius_stats, set_radius_model

__all__ = ["LINKAGE_IDS", "METRIC_IDS", "batched_trees", "fcluster", "linkage",
           "load_radius_model", "pairwise_distances", "radius_stats", "set_radius_model"]

try:  # estimators need scikit-learn
    from ._estimators import AgglomerativeClustering  # noqa: F401
    from ._hdbscan import HDBSCAN  # noqa: F401
    __all__ += ["AgglomerativeClustering", "HDBSCAN"]
except ImportError:  # pragma: no cover - scikit-learn missing
    pass
