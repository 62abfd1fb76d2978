"""Angle subsets for the block algorithms, drop-in for
Python/tigre/utilities/order_subsets.py:31-96 (same modes: None/"ordered",
"random", "random2", "angularDistance")."""
from __future__ import annotations

import numpy as np


def _angular_distance_index(angles):
    a = angles[:, 0]
    idx = np.argsort(a)
    new_index = [idx[0]]
    new_a = [a[idx[0]]]
    rest_a = np.delete(a[idx], 0)
    rest_i = np.delete(idx, 0)
    for i in range(len(rest_a)):
        k = np.argmin(abs(abs(rest_a - new_a[i]) - np.pi / 2))
        new_a.append(rest_a[k])
        new_index.append(rest_i[k])
        rest_a = np.delete(rest_a, k)
        rest_i = np.delete(rest_i, k)
    return np.array(new_index)


def order_subsets(angles, blocksize, mode):
    n = angles.shape[0]
    if blocksize is None or blocksize == 1:
        index = np.arange(n)
        if mode is None or mode == "ordered":
            return list(angles), list(index)
        if mode in ("random", "random2"):
            np.random.shuffle(index)
            return list(angles[index]), list(index)
        if mode == "angularDistance":
            new = _angular_distance_index(angles)
            return list(np.array(angles[new], dtype=np.float32)), list(new)
        raise NameError("mode string not recognized: " + mode)
    nb = (n + blocksize - 1) // blocksize

    def split(order):
        idx = [order[i * blocksize:(i + 1) * blocksize] for i in range(nb - 1)] + [order[(nb - 1) * blocksize:n]]
        return [angles[i] for i in idx], idx

    if mode == "random2":
        order = np.arange(n)
        np.random.shuffle(order)
        return split(order)
    if mode == "angularDistance":
        return split(_angular_distance_index(angles))
    blocks, index = split(np.arange(n, dtype=np.int32))
    if mode is None or mode == "ordered":
        return blocks, index
    if mode == "random":
        order = np.arange(len(index))
        np.random.shuffle(order)
        return [blocks[i] for i in order], [index[i] for i in order]
    raise NameError("mode string not recognized: " + mode)
