"""Seeded synthetic COO tensors for the contraction workloads.

The reference reads FROSTT ``.tns`` files (``mtxTnsIO.cpp:30-65``) and contracts a tensor with a
copy of itself (``sparse_tensor_generator.hpp:4-88``).  No dataset is available offline, so every
workload here is a seeded synthetic tensor with the shapes and value distributions below.

Index distribution ("bounded rank-Zipf"): mode ``m`` draws index ``i`` in ``[0, dim_m)`` with
probability proportional to ``(i + 1) ** -alpha`` (index 0 is the most frequent label), or
uniformly when ``alpha`` is ``None``.  Tuples are drawn in batches; a tuple already drawn is
discarded, so the tensor has exactly ``nnz`` distinct coordinates (FROSTT tensors have no
duplicates, and the reference does not merge duplicates).  The accepted tuples are finally put
in a seeded random order, which is the COO input order the reference sums in.

Everything is numpy ``PCG64`` with a fixed seed, so the same arguments give the same tensor on
any machine with the same numpy major version.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Sequence

import numpy as np


@dataclasses.dataclass
class CooTensor:
    """Host COO tensor in the reference's layout (``tensor.hpp:19-27``).

    ``idx`` is ``uint32[nnz, order]`` with 0-based indices (``hedges_array``), ``vals`` is
    ``float64[nnz]`` (``val_array``) and ``dims`` is ``uint32[order]`` (``dimensions_array``).
    """

    idx: np.ndarray
    vals: np.ndarray
    dims: np.ndarray

    @property
    def order(self) -> int:
        return int(self.idx.shape[1])

    @property
    def nnz(self) -> int:
        return int(self.idx.shape[0])


@dataclasses.dataclass
class Workload:
    """A tensor plus the contraction spec of a meta file (``tensor.hpp:151-173``).

    ``modes`` lists the ``c`` contracted modes first and the free modes after them, exactly like
    the second line of a ``.meta`` file (``4d.meta``).
    """

    name: str
    tensor: CooTensor
    c: int
    modes: list


def _zipf_cdf(dim: int, alpha: float) -> np.ndarray:
    w = np.arange(1, dim + 1, dtype=np.float64) ** (-alpha)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return cdf


def _draw_mode(rng: np.random.Generator, dim: int, alpha: Optional[float], n: int) -> np.ndarray:
    if alpha is None:
        return rng.integers(0, dim, size=n, dtype=np.int64).astype(np.uint32)
    cdf = _zipf_cdf(dim, alpha)
    u = rng.random(n)
    out = np.searchsorted(cdf, u, side="right")
    np.minimum(out, dim - 1, out=out)
    return out.astype(np.uint32)


def random_coo(dims: Sequence[int], nnz: int, alphas: Sequence[Optional[float]], seed: int,
               values: str = "uniform01", max_rounds: int = 64, allow_fewer: bool = False) -> CooTensor:
    """Draw ``nnz`` distinct coordinates (see module docstring) and seeded values.

    ``values``: ``"uniform01"`` U(0,1), ``"normal"`` N(0,1), ``"uniform11"`` U(-1,1).
    With ``allow_fewer``, a distribution too concentrated to yield ``nnz`` distinct tuples within
    ``max_rounds`` draws gives a tensor with the tuples found instead of an error.
    """
    dims = [int(x) for x in dims]
    order = len(dims)
    space = 1
    for dd in dims:
        space *= dd
    if nnz > space:
        raise ValueError(f"nnz {nnz} exceeds the coordinate space {space}")
    if space >= 2 ** 63:
        raise ValueError("coordinate space too large for the generator's 63-bit keys")
    rng = np.random.Generator(np.random.PCG64(seed))
    strides = np.ones(order, dtype=np.uint64)
    for m in range(order - 2, -1, -1):
        strides[m] = strides[m + 1] * np.uint64(dims[m + 1])

    accepted_keys = np.empty(0, dtype=np.uint64)      # in acceptance order
    accepted_sorted = np.empty(0, dtype=np.uint64)
    chunks = []
    need = nnz
    for _ in range(max_rounds):
        if need <= 0:
            break
        draw = max(1024, int(need * 1.25) + 64)
        cols = [_draw_mode(rng, dims[m], alphas[m], draw) for m in range(order)]
        keys = np.zeros(draw, dtype=np.uint64)
        for m in range(order):
            keys += cols[m].astype(np.uint64) * strides[m]
        # first occurrence inside this batch, in draw order
        _, first = np.unique(keys, return_index=True)
        first.sort()
        keys = keys[first]
        # drop tuples accepted in an earlier batch
        if accepted_sorted.size:
            pos = np.searchsorted(accepted_sorted, keys)
            pos = np.minimum(pos, accepted_sorted.size - 1)
            fresh = accepted_sorted[pos] != keys
            keys = keys[fresh]
        keys = keys[:need]
        chunks.append(keys)
        accepted_sorted = np.sort(np.concatenate([accepted_sorted, keys]))
        need -= keys.size
    if need > 0:
        if not allow_fewer:
            raise RuntimeError("generator could not reach the requested number of distinct tuples")
        nnz -= need
    accepted_keys = np.concatenate(chunks)
    perm = rng.permutation(nnz)
    accepted_keys = accepted_keys[perm]
    idx = np.empty((nnz, order), dtype=np.uint32)
    rem = accepted_keys.copy()
    for m in range(order):
        idx[:, m] = (rem // strides[m]).astype(np.uint32)
        rem = rem % strides[m]
    if values == "uniform01":
        vals = rng.random(nnz)
    elif values == "normal":
        vals = rng.standard_normal(nnz)
    elif values == "uniform11":
        vals = rng.uniform(-1.0, 1.0, nnz)
    else:
        raise ValueError(f"unknown value distribution {values!r}")
    return CooTensor(idx=np.ascontiguousarray(idx), vals=np.ascontiguousarray(vals, dtype=np.float64),
                     dims=np.asarray(dims, dtype=np.uint32))


# --- the named workloads ---------------------------------------------------------------------

def uniform3d_50k(seed: int = 0, nnz: int = 50_000) -> Workload:
    """3-D 500x400x300, uniform indices, U(0,1) values, contract modes {0,1}."""
    t = random_coo([500, 400, 300], nnz, [None, None, None], seed, "uniform01")
    return Workload("uniform3d_500x400x300_50k", t, 2, [0, 1, 2])


def zipf4d_3m(seed: int = 1, nnz: int = 3_100_000) -> Workload:
    """4-D 2482x2862x14036x17, per-mode Zipf(1.1), U(0,1) values, contract modes {0,1}."""
    t = random_coo([2482, 2862, 14036, 17], nnz, [1.1, 1.1, 1.1, 1.1], seed, "uniform01")
    return Workload("zipf4d_2482x2862x14036x17_3.1m", t, 2, [0, 1, 2, 3])


def zipf4d_500k(seed: int = 1) -> Workload:
    """The 4-D Zipf workload at 500k nonzeros (same shape, distributions and contraction): the
    small case for profiler captures."""
    w = zipf4d_3m(seed=seed, nnz=500_000)
    return Workload("zipf4d_2482x2862x14036x17_500k", w.tensor, w.c, w.modes)


def skew3d_20m(seed: int = 2, nnz: int = 20_000_000) -> Workload:
    """3-D 12000x9000x28000, Zipf(1.3) on mode 1, uniform modes 0 and 2, N(0,1) values,
    contract modes {0,2} (output indexed by mode 1 x mode 1)."""
    t = random_coo([12000, 9000, 28000], nnz, [None, 1.3, None], seed, "normal")
    return Workload("skew3d_12000x9000x28000_20m", t, 2, [0, 2, 1])


WORKLOADS = {
    "uniform3d_50k": uniform3d_50k,
    "zipf4d_3m": zipf4d_3m,
    "zipf4d_500k": zipf4d_500k,
    "skew3d_20m": skew3d_20m,
}


def describe(name: str) -> str:
    """One line on a named workload: the first sentence of its generator's docstring."""
    doc = " ".join((WORKLOADS[name].__doc__ or name).split())
    return doc.split(". ")[0].rstrip(".")


def batch_member(seed: int) -> Workload:
    """One member of the uneven batch: 3-D or 4-D, dims 64-4096, nnz log-uniform in
    [1k, 200k], Zipf alpha in [0.8, 1.4] on every mode, U(-1,1) values, 1-2 contracted modes
    chosen at random.  ``seed`` selects the member (0..4095 for the 4096-member batch)."""
    rng = np.random.Generator(np.random.PCG64(1_000_003 + seed))
    order = int(rng.integers(3, 5))
    dims = [int(x) for x in rng.integers(64, 4097, size=order)]
    space = math.prod(dims)
    nnz = int(round(math.exp(rng.uniform(math.log(1_000), math.log(200_000)))))
    nnz = min(nnz, space // 4)
    alpha = float(rng.uniform(0.8, 1.4))
    c = int(rng.integers(1, 3))
    modes = [int(x) for x in rng.permutation(order)]
    t = random_coo(dims, nnz, [alpha] * order, seed=2_000_003 + seed, values="uniform11", allow_fewer=True)
    return Workload(f"batch{seed}", t, c, modes)


def batch_members(n: int, procs: int = 0) -> list:
    """Members 0..n-1 of the uneven batch, generated by ``procs`` worker processes (spawned, so a
    process that already uses CUDA may call this)."""
    if procs <= 1:
        return [batch_member(s) for s in range(n)]
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(procs) as pool:
        return pool.map(batch_member, range(n), chunksize=16)


def sizer_member(seed: int, nnz_scale: float = 1.0) -> Workload:
    """One training contraction for the learned sizer: 3-D or 4-D, dims 1k-20k (a 4-D tensor
    keeps one short mode of 8-63, as FROSTT 4-D tensors do), nnz log-uniform in [100k, 5M]
    times ``nnz_scale``, Zipf alpha in [0.8, 1.5] on every mode, U(0,1) values, 1-2 contracted
    modes chosen at random."""
    rng = np.random.Generator(np.random.PCG64(3_000_017 + seed))
    order = int(rng.integers(3, 5))
    dims = [int(x) for x in rng.integers(1_000, 20_001, size=order)]
    if order == 4:
        dims[int(rng.integers(0, 4))] = int(rng.integers(8, 64))
    nnz = int(round(math.exp(rng.uniform(math.log(100_000), math.log(5_000_000)))))
    alpha = float(rng.uniform(0.8, 1.5))
    c = int(rng.integers(1, 3))
    modes = [int(x) for x in rng.permutation(order)]
    nnz = max(2_000, int(nnz * nnz_scale))
    nnz = min(nnz, math.prod(dims) // 4)
    t = random_coo(dims, nnz, [alpha] * order, seed=4_000_037 + seed, values="uniform01", allow_fewer=True)
    return Workload(f"sizer{seed}", t, c, modes)


# --- FROSTT text I/O (host side; the reference uses pigo for this) ----------------------------

def write_tns(path: str, t: CooTensor) -> None:
    """Write 1-based FROSTT text (``i j k ... value`` per line)."""
    with open(path, "w") as f:
        one = t.idx.astype(np.int64) + 1
        for row, v in zip(one, t.vals):
            f.write(" ".join(str(int(x)) for x in row) + " " + repr(float(v)) + "\n")


def read_tns(path: str) -> CooTensor:
    """Read 1-based FROSTT text; dims are the largest label per mode (``mtxTnsIO.cpp:53-57``)."""
    data = np.loadtxt(path, dtype=np.float64, ndmin=2)
    idx = (data[:, :-1].astype(np.int64) - 1).astype(np.uint32)
    vals = data[:, -1].copy()
    dims = (idx.max(axis=0).astype(np.int64) + 1).astype(np.uint32)
    return CooTensor(idx=np.ascontiguousarray(idx), vals=vals, dims=dims)


def write_meta(path: str, c: int, modes: Sequence[int]) -> None:
    """Write a meta file in the reference's format (``4d.meta``): two comment lines, ``c``,
    then the mode list with the contracted modes first."""
    with open(path, "w") as f:
        f.write("#line1: number of contraction modes, c\n")
        f.write("#line2: all the dimensions, such that the first 'c' from the left are the contraction modes\n")
        f.write(f"{c}\n")
        f.write(" ".join(str(int(m)) for m in modes) + "\n")


def read_meta(path: str, order: int):
    """Parse a meta file like ``Tensor::populate_meta_info`` (``tensor.hpp:151-173``)."""
    with open(path) as f:
        lines = f.read().split("\n")
    toks = " ".join(lines[2:]).split()
    c = int(toks[0])
    modes = [int(x) for x in toks[1:1 + order]]
    return c, modes
