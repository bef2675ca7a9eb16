"""Minimal stand-in for the two ``einx`` reductions the reference diagnostics use.

The reference Python solver imports ``einx`` (einx 0.4.3 in its lock file), which is
not installed in this environment. Its Stable Fluids path calls exactly two patterns
(``foilbench_py/core/metrics.py:27,37``):

* ``einx.sum("ny nx [component] -> ny nx", a)``  -> sum over the last axis
* ``einx.mean("[ny nx] component -> component", a)`` -> mean over the first two axes

This module implements only those patterns so the reference can be imported to
generate golden fixtures. Any other pattern raises.
"""

import numpy as np


def sum(pattern, array):  # noqa: A001 - mirrors the einx API name
    if pattern.replace(" ", "") == "nynx[component]->nynx":
        return np.sum(array, axis=-1)
    raise NotImplementedError(pattern)


def mean(pattern, array):
    if pattern.replace(" ", "") == "[nynx]component->component":
        return np.mean(array, axis=(0, 1))
    raise NotImplementedError(pattern)


def dot(pattern, *arrays):
    raise NotImplementedError(pattern)
