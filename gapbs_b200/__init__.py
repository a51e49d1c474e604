"""B200-native engine for the GAP Benchmark Suite's pull-direction PageRank.

The engine is the sm_100a library ``lib/libgapbs_pr.so`` behind the C ABI in
include/pr_gpu.h; graphs come from the host builder ``lib/libgapbs_graph.so``
(include/gapbs_graph.h), which reproduces the reference's graphs exactly.
"""
from .graph import Builder, Graph, GraphBuildError, generate, make_graph
from .pagerank import (K_DAMP, PageRankEngine, PageRankError, PageRankPull, PageRankResult,
                       PersonalizedPageRank, PRVerifier, engine_for, top_scores)

__all__ = ["Builder", "Graph", "GraphBuildError", "generate", "make_graph", "K_DAMP",
           "PageRankEngine", "PageRankError", "PageRankPull", "PageRankResult",
           "PersonalizedPageRank", "PRVerifier", "engine_for", "top_scores"]
