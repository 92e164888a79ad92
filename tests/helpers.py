"""Comparison helpers restating the reference test fixture's checks
(cpp/oneapi/dal/algo/kmeans/test/fixture.hpp:568-720)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_json(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def find_match_centroids(ref, cur):
    """match_map[i] = index of the reference centroid nearest to cur[i]; must be a bijection
    (fixture.hpp:680-706)."""
    ref = np.asarray(ref, np.float64)
    cur = np.asarray(cur, np.float64)
    d = ((cur[:, None, :] - ref[None, :, :]) ** 2).sum(-1)
    m = d.argmin(axis=1)
    assert len(set(m.tolist())) == len(m), "centroid match is not one-to-one"
    return m


def centroid_rel_err(ref, cur, match_map=None):
    """Largest |l - r| / (|l| + |r|) over features, as check_centroid_match_with_rel_tol
    (fixture.hpp:613-662)."""
    ref = np.asarray(ref, np.float64)
    cur = np.asarray(cur, np.float64)
    if match_map is not None:
        ref = ref[match_map]
    diff = np.abs(ref - cur)
    denom = np.abs(ref) + np.abs(cur) + np.finfo(np.float64).tiny
    rel = np.where(diff < np.finfo(np.float64).tiny, 0.0, diff / denom)
    return float(rel.max()) if rel.size else 0.0


def rel_close(val, ref, tol):
    """check_value_with_ref_tol (fixture.hpp:557-564)."""
    m = max(abs(val), abs(ref))
    return m == 0.0 or abs(val - ref) / m < tol


def norm_rel_err(ref, cur):
    """||cur - ref||_F / ||ref||_F."""
    ref = np.asarray(ref, np.float64)
    cur = np.asarray(cur, np.float64)
    den = np.linalg.norm(ref)
    return float(np.linalg.norm(cur - ref) / den) if den > 0 else float(np.linalg.norm(cur))
