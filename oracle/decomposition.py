"""Domain_Decomposition's cost-driven top nodes, restated for one MPI rank.

TEST INFRASTRUCTURE ONLY: the checker for the device decomposition
(tvg_top_nodes with tvg_set_domain_decomposition). Only tests/ use it.

The reference (paths relative to its src/) splits the particles, in
Peano-Hilbert order, into "bunches" -- octree cells along the curve -- and
balances their cost over NTarget targets (NTarget = NTask = the OpenMP
threads on one rank, domain.c:151-156). Restated here step by step:

* find_min_level (domain.c:309-313): level = fmax(2, log(NTarget)/log(8) + 1),
  truncated to int; reset_bunchlist (:281-307) makes the 8^level cells of that
  level, each keyed by the largest short key it can hold.
* fill_new_bunches (:472-531): the particles of a range are counted into
  bunches by their short key (key >> 64); every thread of the team takes its
  static share of the range (GCC's schedule(static) without chunk: the first
  n % T threads one particle more), sums cost_metric (:533-536, the integer
  part of max(1, P.Cost)) into a per-thread float, and the per-thread
  results are added to the bunch in a critical section. This restatement adds
  them in thread order 0 .. T-1; the reference's order is that of the threads'
  arrival, which changes a float sum only when three or more partial sums of
  one bunch are not exactly representable together (above 2^24).
* find_mean_cost (:538-556): Mean_Cost = sum of bunch costs / NTarget,
  Mean_Npart = N / NTarget.
* the loop (:77-107): remove_empty_bunches (:435-470, order kept), sort by key
  with compare_bunches_by_key (descending keys), distribute (:573-628: sort
  by cost descending, give each bunch to the target furthest below the mean
  cost, sort by key again, Split_Idx[t] = the costliest bunch of target t
  starting from bunch index t), find_global_imbalances (:630-652); stop when
  the cost imbalance is below DOMAIN_IMBAL_CEIL and the particle imbalance
  below Part_Alloc_Factor - 1, or after N_SHORT_TRIPLETS - MIN_LEVEL + 1
  rounds; else mark_bunches_to_split (:654-676) and make_new_bunchlist
  (:374-406) with split_bunch (:408-433).
* transform_bunches_into_top_nodes (:220-250): top nodes in the final order
  (descending keys) with Level, First_Part and Npart of their bunch.

Both sorts are the C library's qsort with the reference's comparators, called
through ctypes, so that equal costs keep whatever order qsort gives them.
"""
from __future__ import annotations

import ctypes as C
import ctypes.util
import math

import numpy as np

MIN_LEVEL = 2                 # domain.c:3
N_SHORT_BITS = 64             # peano.h
N_SHORT_TRIPLETS = N_SHORT_BITS // 3
INT_MAX = 2 ** 31 - 1


class Bunch(C.Structure):
    """struct Bunch_Node (domain.h:29-38), the members the loop uses."""
    _fields_ = [("Key", C.c_uint64), ("Target", C.c_int), ("Level", C.c_int),
                ("First_Part", C.c_int), ("Npart", C.c_uint64), ("Cost", C.c_float),
                ("Modify", C.c_int)]


_CMP = C.CFUNCTYPE(C.c_int, C.POINTER(Bunch), C.POINTER(Bunch))


def _by_key(a, b):            # compare_bunches_by_key (domain.c:678-684)
    x, y = a.contents.Key, b.contents.Key
    return int(x < y) - int(x > y)


def _by_cost(a, b):           # compare_bunches_by_cost (domain.c:686-692)
    x, y = a.contents.Cost, b.contents.Cost
    return int(x < y) - int(x > y)


_cmp_key, _cmp_cost = _CMP(_by_key), _CMP(_by_cost)
_libc = C.CDLL(ctypes.util.find_library("c"))
_libc.qsort.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, _CMP]
_libc.qsort.restype = None


def _qsort(D, cmp):
    arr = (Bunch * len(D))(*D)
    _libc.qsort(C.cast(arr, C.c_void_p), len(D), C.sizeof(Bunch), cmp)
    return [Bunch.from_buffer_copy(arr[i]) for i in range(len(D))]


def min_level(ntarget):
    """find_min_level (domain.c:309-313)."""
    return int(max(MIN_LEVEL, math.log(ntarget) / math.log(8) + 1))


def static_chunks(n, nthreads):
    """[start, end) of every thread's share of n iterations, as GCC expands
    `#pragma omp for` without a schedule clause."""
    q, r = divmod(n, nthreads)
    out = []
    for t in range(nthreads):
        if t < r:
            s = (q + 1) * t
            out.append((s, s + q + 1))
        else:
            s = q * t + r
            out.append((s, s + q))
    return out


def fill(D, first_bunch, nb, first_part, npart, key_hi, metric, nthreads):
    """fill_new_bunches (domain.c:472-531) for bunches first_bunch ..
    first_bunch + nb - 1 and particles first_part .. first_part + npart - 1."""
    keys = np.array([D[first_bunch + i].Key for i in range(nb)], np.uint64)
    for i in range(nb):
        D[first_bunch + i].Npart = 0
        D[first_bunch + i].Cost = 0.0
        D[first_bunch + i].First_Part = INT_MAX
    partial = []
    for s, e in static_chunks(npart, nthreads):
        a, b = first_part + s, first_part + e
        # bunch of each particle: the first with Key >= the particle's key
        run = np.searchsorted(keys, key_hi[a:b], side="left")
        cnt = np.zeros(nb, np.int64)
        cost = np.zeros(nb, np.float32)
        first = np.full(nb, INT_MAX, np.int64)
        if b > a:
            for k in np.unique(run):
                sel = np.nonzero(run == k)[0]
                cnt[k] = len(sel)
                # sequential float sum of the thread's particles in bunch k
                cost[k] = np.cumsum(metric[a + sel].astype(np.float32), dtype=np.float32)[-1]
                first[k] = a + sel[0]
        partial.append((cnt, cost, first))
    for cnt, cost, first in partial:               # the critical section, thread order
        for i in range(nb):
            d = D[first_bunch + i]
            d.Npart += int(cnt[i])
            d.Cost = float(np.float32(d.Cost) + cost[i])
            d.First_Part = int(min(d.First_Part, first[i]))


def decompose(key_hi, cost, ntask, part_alloc_factor=1.1, imbal_ceil=0.05):
    """Top nodes of Domain_Decomposition on one rank for NTask = ntask.

    key_hi: the short keys (high 64 bits of the standard keys) in sorted
    order; cost: P.Cost in the same order. Returns a list of (Key, Level,
    First_Part, Npart) in the final top-node order, and the number of rounds.
    """
    key_hi = np.ascontiguousarray(key_hi, np.uint64)
    n = len(key_hi)
    ntarget = ntask if ntask < 65 else 1
    nthreads = ntask
    # cost_metric: (unsigned int) fmax(1, P.Cost)
    metric = np.floor(np.maximum(1.0, np.asarray(cost, np.float64))).astype(np.uint64)
    lvl = min_level(ntarget)
    nb = 8 ** lvl
    shift = 3 * lvl
    base = (0xFFFFFFFFFFFFFFFF >> shift)
    D = []
    for i in range(nb):                           # reset_bunchlist
        b = Bunch()
        b.Key = ((i << (64 - shift)) & 0xFFFFFFFFFFFFFFFF) | base
        b.Level, b.Npart, b.First_Part, b.Target, b.Modify = lvl, 0, INT_MAX, -1, 0
        D.append(b)
    fill(D, 0, nb, 0, n, key_hi, metric, nthreads)
    mean_cost = sum(float(d.Cost) for d in D) / ntarget       # find_mean_cost
    mean_npart = float(n) / ntarget
    cnt = 0
    while True:
        D = [d for d in D if d.Npart != 0]                     # remove_empty_bunches
        D = _qsort(D, _cmp_key)
        # distribute
        tcost = np.zeros(ntarget, np.float32)
        tnpart = np.zeros(ntarget, np.int64)
        D = _qsort(D, _cmp_cost)
        for d in D:
            task, maxd = 0, 0.0
            for j in range(ntarget):
                delta = mean_cost - float(tcost[j])
                if delta > maxd:
                    task, maxd = j, delta
            tcost[task] = np.float32(tcost[task] + np.float32(d.Cost))
            tnpart[task] += d.Npart
            d.Target = -task - 1
        D = _qsort(D, _cmp_key)
        split = list(range(ntarget))
        for i, d in enumerate(D):
            task = -(d.Target + 1)
            if d.Cost > D[split[task]].Cost:
                split[task] = i
        # find_global_imbalances
        cost_imbal = max(abs(float(c) - mean_cost) / mean_cost for c in tcost)
        mem_imbal = max(abs(float(m) - mean_npart) / mean_npart for m in tnpart)
        if cost_imbal < imbal_ceil and mem_imbal < part_alloc_factor - 1:
            break
        if cnt > N_SHORT_TRIPLETS - MIN_LEVEL:
            break
        cnt += 1
        for t in range(ntarget):                              # mark_bunches_to_split
            j = split[t]
            if j >= 0 and D[j].Level != N_SHORT_TRIPLETS:
                D[j].Modify = 1
        old = len(D)                                          # make_new_bunchlist
        for i in range(old):
            if D[i].Modify == 0:
                continue
            first_new = len(D)
            for c in range(8):                                # split_bunch
                b = Bunch()
                b.Level = D[i].Level + 1
                sh = N_SHORT_BITS - 3 * b.Level
                mask = (0x7 << sh) & 0xFFFFFFFFFFFFFFFF
                b.Key = (D[i].Key & ~mask & 0xFFFFFFFFFFFFFFFF) | ((c << sh) & 0xFFFFFFFFFFFFFFFF)
                b.Npart, b.First_Part, b.Target, b.Modify = 0, INT_MAX, -1, 0
                D.append(b)
            fill(D, first_new, 8, D[i].First_Part, D[i].Npart, key_hi, metric, nthreads)
            D[i].Npart = 0
    return [(d.Key, d.Level, d.First_Part, int(d.Npart)) for d in D], cnt
