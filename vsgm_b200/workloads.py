"""Seeded synthetic workloads (the reference's Friendster/SNAP inputs are replaced
by generators with fixed seeds; every graph is written in the reference .bin
layout by write_csr_bin when a file is wanted).

    triangle_rmat16()        -kc 3 on R-MAT scale 16, edge factor 16, seed 1
    patterns_rmat22()        -kc 4, -p 1, -p 2 on R-MAT scale 22, edge factor 16, seed 2
    chung_lu_views(...)      16 Chung-Lu views: exponent U[2.1, 2.8], 1e5..1e7 edges
                             (log-uniform), max expected degree 1e4, seed 3
    random_patterns(...)     64 connected patterns of 3..6 vertices, p = 0.5, seed 3
    social_chung_lu()        65M vertices, ~1.8B edges, exponent 2.2, max degree 5000, seed 5
"""
import math

import numpy as np

from . import gen_chung_lu, gen_rmat, plan_clique, plan_pattern, plan_query_bits, random_pattern
from .workload_rng import stream_uniform

RMAT_ABC = (0.57, 0.19, 0.19)


def triangle_rmat16(threads=0):
    return gen_rmat(16, 16, *RMAT_ABC, seed=1, threads=threads), [plan_clique(3)]


def patterns_rmat22(threads=0, scale=22):
    g = gen_rmat(scale, 16, *RMAT_ABC, seed=2, threads=threads)
    return g, [plan_clique(4), plan_pattern(1), plan_pattern(2)]


def chung_lu_specs(n=16, seed=3, e_min=1e5, e_max=1e7, avg_degree=16):
    """(vertices, target edges, exponent) of every view, drawn from stream `seed`."""
    specs = []
    for i in range(n):
        gamma = 2.1 + 0.7 * stream_uniform(seed, 2 * i)
        edges = int(round(math.exp(math.log(e_min) + (math.log(e_max) - math.log(e_min)) * stream_uniform(seed, 2 * i + 1))))
        V = max(1000, 2 * edges // avg_degree)
        specs.append((V, edges, gamma))
    return specs


def chung_lu_views(n=16, seed=3, e_min=1e5, e_max=1e7, max_degree=10_000, threads=0):
    return [gen_chung_lu(V, E, gamma, max_degree, seed=seed * 1000 + i, threads=threads)
            for i, (V, E, gamma) in enumerate(chung_lu_specs(n, seed, e_min, e_max))]


def random_patterns(n=64, seed=3, n_min=3, n_max=6, p=0.5):
    out, ctr = [], 0
    for _ in range(n):
        k, bits, ctr = random_pattern(seed=seed, counter=ctr, n_min=n_min, n_max=n_max, p=p)
        out.append(plan_query_bits(k, bits))
    return out


def social_chung_lu(threads=0, V=65_000_000, edges=1_800_000_000):
    return gen_chung_lu(V, edges, 2.2, 5000, seed=5, threads=threads)
