"""Synthetic workloads with the shapes of the reference's benchmark configurations.

The reference benchmarks on no public dataset; every workload here is seeded
synthetic data from the Hardy-Weinberg/planted generator of libepik2
(epik2_generate_hwe).  Seeds: workload c uses seed 1000 + c; dataset d of a
multi-dataset workload uses seed (1000 + c) * 1000 + d.
"""
import math
import random

PLAIN_SMALL = dict(name="plain-small 512 SNPs x 2048 samples", seed=1001, n_snps=512, n_samples=2048, n_cases=1024,
                   maf=(0.05, 0.5), planted=[(17, 203, 411)], effects=[0.8])
PLAIN_LARGE = dict(name="plain-large 4096 SNPs x 16384 samples", seed=1002, n_snps=4096, n_samples=16384,
                   n_cases=8192, maf=(0.05, 0.5), planted=[(17, 203, 411)], effects=[0.8])
PRECISION = dict(name="precision 2048 SNPs x 8192 samples", seed=1003, n_snps=2048, n_samples=8192, n_cases=4096,
                 maf=(0.01, 0.5), planted=[(17, 203, 411), (64, 777, 1500), (300, 1024, 2000)],
                 effects=[0.6, 0.7, 0.8])

CONFIGS = {"plain-small": PLAIN_SMALL, "plain-large": PLAIN_LARGE, "precision": PRECISION}


def generate(cfg, n_snps=None):
    """Genotypes and phenotype of a workload (optionally only its first n_snps columns)."""
    from . import generate_hwe
    g, ph = generate_hwe(cfg["seed"], cfg["n_samples"], cfg["n_snps"], cfg["n_cases"], cfg["maf"], cfg["planted"],
                         cfg["effects"])
    if n_snps is not None and n_snps < cfg["n_snps"]:
        g = g[:, :n_snps].copy()
    return g, ph


def batched_specs(n_datasets=96, seed=1004):
    """96 independent datasets: SNPs log-uniform in [128,1536], samples log-uniform in
    [1000,12000], case fraction uniform in [0.3,0.7], one planted triplet each."""
    rng = random.Random(seed)
    specs = []
    for d in range(n_datasets):
        m = int(round(math.exp(rng.uniform(math.log(128), math.log(1536)))))
        s = int(round(math.exp(rng.uniform(math.log(1000), math.log(12000)))))
        frac = rng.uniform(0.3, 0.7)
        planted = (m // 7, m // 2, m - 3)
        specs.append(dict(name=f"batched-{d}", seed=seed * 1000 + d, n_snps=m, n_samples=s,
                          n_cases=int(round(frac * s)), maf=(0.05, 0.5), planted=[planted], effects=[0.8]))
    return specs


SERVING = dict(
    resident=[
        dict(name="resident-A 1024 SNPs x 8192 samples", seed=1005000, n_snps=1024, n_samples=8192, n_cases=4096,
             maf=(0.05, 0.5), planted=[(17, 203, 411)], effects=[0.8]),
        dict(name="resident-B 3072 SNPs x 4096 samples", seed=1005001, n_snps=3072, n_samples=4096, n_cases=2048,
             maf=(0.05, 0.5), planted=[(17, 203, 411)], effects=[0.8]),
    ],
    rate_per_s=20.0, duration_s=60.0, replicates=(16, 1000), upload_frac=0.10, upload_snps=(256, 768), seed=1005)
