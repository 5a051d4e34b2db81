"""Ensemble generation and partition formats.

Drop-in for MyML/MyML/utils/partition.py: ``generateEnsemble`` (:88-124) and
``convertClusterStringToIndex`` (:73-86).  All partitions of an ensemble are
fitted together in one batched GPU pass (``kmeans_ensemble``); the random
draws (k per partition with np.random.randint, the initial sample with
random.sample) are made on the host in the reference's order, so a seeded
run reproduces the reference's ensemble exactly.
"""
import random

import numpy as np

from ..cluster.KMeans import kmeans_ensemble


def convertClusterStringToIndex(partition):
    """Label array -> list of member-index arrays (uint64, ascending), one per
    distinct label in ascending label order (MyML/MyML/utils/partition.py:73-86)."""
    partition = np.asarray(partition)
    order = np.argsort(partition, kind="stable")
    labels, starts = np.unique(partition[order], return_index=True)
    bounds = list(starts) + [partition.size]
    return [order[bounds[c]:bounds[c + 1]].astype(np.uint64) for c in range(labels.size)]


def draw_ensemble_params(n_samples, n_clusters, npartitions):
    """The host random draws of generateEnsemble + K_Means.fit, in order."""
    ks, inits = [], []
    cluster_range = isinstance(n_clusters, list) and n_clusters[0] != n_clusters[1]
    for _ in range(npartitions):
        if cluster_range:
            k = int(np.random.randint(n_clusters[0], n_clusters[1]))
        elif isinstance(n_clusters, list):
            k = int(n_clusters[0])
        else:
            k = int(n_clusters)
        ks.append(k)
        inits.append(random.sample(range(n_samples), k))
    return ks, inits


def generate_ensemble_labels(data, n_clusters=20, npartitions=30, iters=3, label_mode="cuda",
                             centroid_mode="numba", tol=1e-4, stream=None):
    """The ensemble as a device label matrix (npartitions x n int32), the
    format the co-association build consumes directly."""
    n = int(data.shape[0])
    ks, inits = draw_ensemble_params(n, n_clusters, npartitions)
    labels, _, _, _, _ = kmeans_ensemble(data, ks, inits, max_iter=iters, tol=tol,
                                         label_mode=label_mode, centroid_mode=centroid_mode,
                                         stream=stream)
    return labels, ks


def generateEnsemble(data, generator, n_clusters=20, npartitions=30, iters=3):
    """MyML/MyML/utils/partition.py:88-124.  ``generator`` is a K_Means whose
    label/centroid modes and tol are used; returns the list-of-clusters
    ensemble of the reference."""
    generator.max_iter = iters
    labels, _ = generate_ensemble_labels(
        data, n_clusters, npartitions, iters,
        label_mode=getattr(generator, "_label_mode", "cuda"),
        centroid_mode=getattr(generator, "_centroid_mode", "numba"),
        tol=getattr(generator, "tol", 1e-4))
    L = labels.cpu().numpy()
    return [convertClusterStringToIndex(L[p]) for p in range(L.shape[0])]
