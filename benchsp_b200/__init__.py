"""benchsp_b200 — B200-native (sm_100a) SpMV/SpMM library with the operator
surface of jiajun-c/benchsp.  The compute path is libbspmv.so (hand-written
CUDA behind the C ABI in include/bsp.h); this package is its Python host API.
"""
from ._lib import BspError, lib  # noqa: F401
from .api import (GatherTileMatrix, gather_probe, gen_diffusion3d, gen_block_laplace3d, MtxFile, read_mtx, write_mtx, reorder_rcm, reorder_rcm_host, permute_csr, permute_csr_host, reorder_similarity, reorder_similarity_host, permute_rows_csr, permute_rows_csr_host, choose_spmm_host, SpmvPlan, tune_spmv, matrix_key, tune_cache_clear, BatchPlan, gen_batch, gen_banded, SpmmPlan, SmatMatrix, gen_graph, spmm_csr, CgSolver, blockinfo, BcsrMatrix, BsrMatrix, BsrScaledMatrix, DaspMatrix, DbsrMatrix, csr2bcsr, csr2dasp, HostCSR, csr2bsr, csr2dbsr, csr_merge_workspace_bytes, csr_spmv,  # noqa: F401
                  csr_spmv_merge, gen_laplace2d, gen_poisson3d, gen_powerlaw, gen_random_bsr,
                  gen_stencil27, gen_uniform)

__all__ = ["BspError", "lib", "GatherTileMatrix", "gather_probe", "gen_diffusion3d", "gen_block_laplace3d", "MtxFile", "read_mtx", "write_mtx", "reorder_rcm", "reorder_rcm_host", "permute_csr", "permute_csr_host", "reorder_similarity", "reorder_similarity_host", "permute_rows_csr", "permute_rows_csr_host", "choose_spmm_host", "SpmvPlan", "tune_spmv", "matrix_key", "tune_cache_clear", "BatchPlan", "gen_batch", "gen_banded", "SpmmPlan", "SmatMatrix", "gen_graph", "spmm_csr", "CgSolver", "blockinfo", "BcsrMatrix", "csr2bcsr", "DaspMatrix", "csr2dasp", "BsrMatrix", "BsrScaledMatrix", "DbsrMatrix", "csr2dbsr", "HostCSR", "csr2bsr", "csr_merge_workspace_bytes", "csr_spmv",
           "csr_spmv_merge", "gen_laplace2d", "gen_poisson3d", "gen_powerlaw", "gen_random_bsr",
           "gen_stencil27", "gen_uniform"]
