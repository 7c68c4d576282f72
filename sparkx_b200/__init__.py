"""B200-native PKT k-truss decomposition (drop-in for SparX's ``k_truss`` PKT path).

Public surface mirrors the reference's ``AlgoPKT`` (``src/k_truss/pkt.rs:29-123``):
``AlgoPKT.new(graph)``, ``trussness(e)``, ``k_trusses()``, ``drop_cache()``; the
graph is a memory-mapped CSR like ``GraphMemoryMap`` (``src/graph/mod.rs:365-378``).
``AlgoBurkhardtEtAl`` (the default ``k_truss``), ``Triangles``,
``ClusteringCoefficient`` and the k-core ``AlgoLiuEtAl`` run on the same GPU engine.
"""
from .graph import GraphMemoryMap  # noqa: F401
from .pkt import (AlgoBurkhardtEtAl, AlgoLiuEtAl, AlgoPKT, ClusteringCoefficient,  # noqa: F401
                  PktError, PktOptions, PktStats, Triangles)

__all__ = ["GraphMemoryMap", "AlgoPKT", "AlgoBurkhardtEtAl", "AlgoLiuEtAl", "Triangles",
           "ClusteringCoefficient", "PktOptions", "PktStats", "PktError"]
