"""onedal_b200 -- B200-native k-means Lloyd (dense) behind oneDAL's train/infer surface.

``onedal_b200.kmeans`` mirrors ``oneapi::dal::kmeans``; the compute is the CUDA
library ``onedal_b200/lib/libonedal_b200_kmeans.so`` (C ABI:
include/onedal_b200_kmeans.h), built by ``python -m onedal_b200.build``.
"""
from . import kmeans  # noqa: F401

__version__ = "0.1.0"
