"""ctypes binding to libswgpu.so, the B200 engine for MNHN-Tree-Tools'
all-pairs Smith-Waterman neighbourhood path.

The library is C (include/swgpu.h, include/mnhn_dropin.h); this module is a
thin host-side wrapper for tests, benchmarks and Python callers.  Every call
goes to the CUDA path; nothing here computes a distance on the CPU.  Calls
raise ``SwgpuError`` carrying the C status when the library reports one, and
importing fails loudly when the shared library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

PKG_ROOT = Path(__file__).resolve().parent.parent          # mnhn-tree-tools_b200/
LIB_PATH = PKG_ROOT / "lib" / "libswgpu.so"
BIN_DIR = PKG_ROOT / "bin"
INCLUDE_DIR = PKG_ROOT.parent / "include"

STATUS = {0: "SWE_OK", 1: "SWE_ERR_INVALID", 2: "SWE_ERR_CUDA", 3: "SWE_ERR_OOM",
          4: "SWE_ERR_NO_DEVICE", 5: "SWE_ERR_TIMEOUT", 6: "SWE_ERR_RERUN", 7: "SWE_ERR_STATE",
          8: "SWE_ERR_IO", 9: "SWE_ERR_SWEEP"}


class SwgpuError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def build(force: bool = False) -> None:
    """Compile libswgpu.so and the command-line tools (nvcc, sm_100a)."""
    if force or not LIB_PATH.exists():
        subprocess.run(["make", "-s", "-j8", "-C", str(PKG_ROOT)], check=True)


# ---------------------------------------------------------------------------
# structures (include/mnhn_types.h, include/swgpu.h)
# ---------------------------------------------------------------------------
class Dataset(C.Structure):
    _fields_ = [("sequences", C.POINTER(C.c_char_p)), ("sequence_lengths", C.POINTER(C.c_size_t)),
                ("binary_sequences", C.c_void_p), ("n_values", C.c_int), ("values", C.c_void_p),
                ("n_dimensions", C.c_int), ("max_sequence_length", C.c_size_t)]


class Cluster(C.Structure):
    _fields_ = [("members", C.POINTER(C.c_int)), ("n_members", C.c_int), ("id", C.c_int)]


class SplitSet(C.Structure):
    _fields_ = [("n_clusters", C.c_int), ("clusters", C.POINTER(Cluster))]


class Opts(C.Structure):
    _fields_ = [("device", C.c_int), ("sat_limit", C.c_int), ("packs_per_block", C.c_int),
                ("threads", C.c_int), ("inject_timeout", C.c_int),
                ("threshold_path", C.c_int), ("kmer_batch_kb", C.c_int), ("max_w", C.c_int),
                ("dbscan_replay", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("n_sequences", C.c_int64), ("n_fast", C.c_int64), ("n_exceptional", C.c_int64),
                ("unique_pairs", C.c_int64), ("cells", C.c_double), ("tile_cells", C.c_double),
                ("reruns", C.c_int64), ("n_tiles", C.c_int64), ("ms_score_pass", C.c_double),
                ("ms_fast_kernel", C.c_double), ("ms_last_neighbors", C.c_double),
                ("last_neighbor_launches", C.c_int64),
                ("dist_bytes", C.c_int), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
                ("kernel_launches", C.c_int64), ("ms_last_batch", C.c_double), ("ms_last_replay", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PrefilterStats(C.Structure):
    _fields_ = [("candidates", C.c_int64), ("tiles_kept", C.c_int64), ("tiles_all", C.c_int64),
                ("tile_cells", C.c_double), ("ms_embed", C.c_double), ("ms_candidates", C.c_double),
                ("ms_layout", C.c_double), ("ms_score", C.c_double), ("ms_total", C.c_double),
                ("fallback_full", C.c_int), ("ms_groups", C.c_double), ("ms_marks", C.c_double),
                ("ms_upload", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Margins(C.Structure):
    _fields_ = [("n", C.c_int), ("upper", C.c_int * 8), ("margin", C.c_float * 8)]

    @staticmethod
    def of(m):
        """A float (one margin for every pair) or a list of (upper, margin)
        buckets by the pair's longer length (the last upper is ignored)."""
        if isinstance(m, (int, float)):
            m = [(0, float(m))]
        t = Margins()
        t.n = len(m)
        for i, (u, v) in enumerate(m):
            t.upper[i] = int(u)
            t.margin[i] = float(v)
        return t


class TuneResult(C.Structure):
    _fields_ = [("packs_per_block", C.c_int), ("threads", C.c_int), ("max_w", C.c_int), ("from_cache", C.c_int),
                ("candidates", C.c_int), ("sample", C.c_int), ("sample_cells", C.c_double),
                ("ms_default", C.c_double), ("ms_best", C.c_double), ("key", C.c_char * 160)]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["key"] = self.key.decode()
        return d


class SweepResult(C.Structure):
    _fields_ = [("status", C.c_int), ("truncated", C.c_int), ("steps", C.c_int), ("n_layers", C.c_int),
                ("layers", C.POINTER(SplitSet)), ("log", C.c_void_p), ("done_ms", C.c_double)]


DBSCANNER = C.CFUNCTYPE(SplitSet, Dataset, C.c_float, C.c_int)
TEXT_SINK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_size_t, C.c_void_p)


class KmerFrequencies(C.Structure):
    # kmers.h:17-21
    _fields_ = [("frequencies", C.POINTER(C.POINTER(C.c_short))), ("n_kmers", C.c_size_t),
                ("n_seq", C.c_size_t)]

class DataShape(C.Structure):
    # dataset.h:37-40 (kmer2pca.c:20-23 declares the same struct)
    _fields_ = [("n_features", C.c_size_t), ("n_samples", C.c_size_t)]


class PcaInfo(C.Structure):
    # swgpu.h: swe_pca_info
    _fields_ = [("exact", C.c_int), ("h2d_bytes", C.c_int64), ("ms_upload", C.c_double),
                ("ms_covariance", C.c_double), ("ms_gram", C.c_double), ("ms_eigen", C.c_double),
                ("ms_project", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# Every symbol the public headers declare (checked by the CPU test suite).
EXPORTS = [
    # include/swgpu.h
    "swe_strerror", "swe_create", "swe_destroy", "swe_last_error", "swe_upload",
    "swe_score_all_pairs", "swe_copy_distances", "swe_neighbors", "swe_dbscan", "swe_adaptive",
    "swe_score_one_to_many", "swe_score_pairs", "swe_get_stats", "swe_free", "swe_dbscan_bitmap",
    "swe_dbscan_bitmaps_device",
    "swe_measure_mix_peak", "swe_timer_start", "swe_timer_stop", "swe_score_pairs_noalloc",
    "swe_upload_sets", "swe_set_count", "swe_copy_set_distances", "swe_neighbors_set", "swe_dbscan_set",
    "swe_adaptive_set", "swe_adaptive_sets", "swe_free_sweep_results",
    "swe_kmer_features", "swe_prefilter_init", "swe_prefilter_param_count", "swe_prefilter_params",
    "swe_prefilter_loss_grad", "swe_prefilter_train", "swe_prefilter_embed", "swe_prefilter_pair_dist",
    "swe_gemm_bf16", "swe_prefilter_set_embeddings", "swe_score_prefiltered",
    "swe_kmer_count", "swe_kmer_counts", "swe_kmer_tsv", "swe_upload_points", "swe_adaptive_matrix",
    "swe_set_partition", "swe_distance_bytes", "swe_distance_copy", "swe_lpt_partition", "swe_capped_linkage", "swe_cost_order",
    "swe_pca_covariance", "swe_pca_eigen", "swe_pca_eigen_gpu", "swe_pca_project", "swe_pca",
    "swe_autotune", "swe_copy_set_rows", "swe_partition_bytes", "swe_partition_pack", "swe_partition_unpack",
    # include/mnhn_dropin.h
    "score", "dataset_from_fasta", "free_sequences_from_dataset", "dbscan_SW", "adaptive_dbscan",
    "store_split_set", "read_split_set", "create_single_cluster_file", "create_cluster_files",
    "data_not_in_clusters", "intersection_of_clusters", "generate_split_set_relation",
    "free_split_set_and_associated_clusters", "swgpu_last_dropin_status",
    "frequencies_from_dataset", "write_kmer_base", "free_kmer_frequencies", "dbscan_L1", "dbscan_L2",
    "shape_from_kmer_file", "load_kmer_from_file_into_dataset", "free_values_from_dataset", "free_dataset",
    "create_single_cluster_file_with_values", "create_cluster_files_with_values", "swe_read_feature_table",
]

_lib = None


def lib():
    """Load libswgpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {PKG_ROOT}`")
        L = C.CDLL(str(LIB_PATH))
        L.swe_strerror.restype = C.c_char_p
        L.swe_strerror.argtypes = [C.c_int]
        L.swe_create.restype = C.c_int
        L.swe_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(Opts)]
        L.swe_destroy.argtypes = [C.c_void_p]
        L.swe_last_error.restype = C.c_char_p
        L.swe_last_error.argtypes = [C.c_void_p]
        L.swe_upload.restype = C.c_int
        L.swe_upload.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.swe_score_all_pairs.restype = C.c_int
        L.swe_score_all_pairs.argtypes = [C.c_void_p]
        L.swe_copy_distances.restype = C.c_int
        L.swe_copy_distances.argtypes = [C.c_void_p, C.c_void_p]
        L.swe_neighbors.restype = C.c_int
        L.swe_neighbors.argtypes = [C.c_void_p, C.c_float, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.swe_dbscan.restype = C.c_int
        L.swe_dbscan.argtypes = [C.c_void_p, C.c_float, C.c_int, C.POINTER(SplitSet)]
        L.swe_adaptive.restype = C.c_int
        L.swe_adaptive.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_int, C.c_char_p, C.c_void_p,
                                   C.POINTER(C.POINTER(SplitSet)), C.POINTER(C.c_int)]
        L.swe_upload_sets.restype = C.c_int
        L.swe_upload_sets.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.swe_set_count.restype = C.c_int
        L.swe_set_count.argtypes = [C.c_void_p]
        L.swe_copy_set_distances.restype = C.c_int
        L.swe_copy_set_distances.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.swe_partition_bytes.restype = C.c_int64
        L.swe_partition_bytes.argtypes = [C.c_void_p, C.c_int]
        L.swe_partition_pack.restype = C.c_int
        L.swe_partition_pack.argtypes = [C.c_void_p, C.c_void_p]
        L.swe_partition_unpack.restype = C.c_int
        L.swe_partition_unpack.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_int64]
        L.swe_autotune.restype = C.c_int
        L.swe_autotune.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_char_p, C.c_int,
                                   C.POINTER(TuneResult)]
        L.swe_copy_set_rows.restype = C.c_int
        L.swe_copy_set_rows.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.swe_neighbors_set.restype = C.c_int
        L.swe_neighbors_set.argtypes = [C.c_void_p, C.c_int, C.c_float, C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p)]
        L.swe_dbscan_set.restype = C.c_int
        L.swe_dbscan_set.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_int, C.POINTER(SplitSet)]
        L.swe_adaptive_set.restype = C.c_int
        L.swe_adaptive_set.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_int, C.c_char_p,
                                       C.c_void_p, C.POINTER(C.POINTER(SplitSet)), C.POINTER(C.c_int)]
        L.swe_adaptive_sets.restype = C.c_int
        L.swe_adaptive_sets.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_int, C.c_int, C.c_char_p,
                                        C.POINTER(SweepResult)]
        L.swe_free_sweep_results.argtypes = [C.POINTER(SweepResult), C.c_int]
        L.swe_kmer_features.restype = C.c_int
        L.swe_kmer_features.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.swe_prefilter_init.restype = C.c_int
        L.swe_prefilter_init.argtypes = [C.c_void_p, C.c_uint64]
        L.swe_prefilter_param_count.restype = C.c_int64
        L.swe_prefilter_param_count.argtypes = []
        L.swe_prefilter_params.restype = C.c_int
        L.swe_prefilter_params.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.swe_prefilter_loss_grad.restype = C.c_int
        L.swe_prefilter_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                              C.POINTER(C.c_float), C.c_void_p]
        L.swe_prefilter_train.restype = C.c_int
        L.swe_prefilter_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                                          C.c_int, C.c_float, C.c_float, C.c_uint64, C.c_float, C.c_float,
                                          C.c_void_p]
        L.swe_prefilter_embed.restype = C.c_int
        L.swe_prefilter_embed.argtypes = [C.c_void_p, C.c_void_p]
        L.swe_prefilter_pair_dist.restype = C.c_int
        L.swe_prefilter_pair_dist.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        L.swe_prefilter_set_embeddings.restype = C.c_int
        L.swe_prefilter_set_embeddings.argtypes = [C.c_void_p, C.c_void_p]
        L.swe_score_prefiltered.restype = C.c_int
        L.swe_score_prefiltered.argtypes = [C.c_void_p, C.c_float, C.POINTER(Margins), C.c_int,
                                            C.POINTER(PrefilterStats)]
        L.swe_gemm_bf16.restype = C.c_int
        L.swe_gemm_bf16.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                    C.c_int, C.c_void_p]
        L.swe_score_one_to_many.restype = C.c_int
        L.swe_score_one_to_many.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t, C.c_void_p]
        L.swe_score_pairs.restype = C.c_int
        L.swe_score_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        L.swe_get_stats.restype = C.c_int
        L.swe_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.swe_free.argtypes = [C.c_void_p]
        L.swe_measure_mix_peak.restype = C.c_int
        L.swe_measure_mix_peak.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.swe_timer_start.restype = C.c_int
        L.swe_timer_start.argtypes = [C.c_void_p]
        L.swe_timer_stop.restype = C.c_int
        L.swe_timer_stop.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.swe_score_pairs_noalloc.restype = C.c_int
        L.swe_score_pairs_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                              C.c_void_p, C.c_int, C.c_void_p]
        L.swe_dbscan_bitmaps_device.restype = C.c_int
        L.swe_dbscan_bitmaps_device.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                                C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.POINTER(SplitSet)]
        L.swe_dbscan_bitmap.restype = C.c_int
        L.swe_dbscan_bitmap.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(SplitSet)]
        L.score.restype = C.c_uint
        L.score.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t, C.c_size_t, C.c_void_p]
        L.dbscan_SW.restype = SplitSet
        L.dbscan_SW.argtypes = [Dataset, C.c_float, C.c_int]
        L.adaptive_dbscan.restype = None
        L.adaptive_dbscan.argtypes = [C.c_void_p, Dataset, C.c_float, C.c_float, C.c_int, C.c_char_p, C.c_int]
        L.free_split_set_and_associated_clusters.argtypes = [SplitSet]
        L.store_split_set.argtypes = [C.c_char_p, SplitSet]
        L.read_split_set.restype = SplitSet
        L.read_split_set.argtypes = [C.c_char_p]
        L.swgpu_last_dropin_status.restype = C.c_int
        L.swe_set_partition.restype = C.c_int
        L.swe_set_partition.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.swe_distance_bytes.restype = C.c_int64
        L.swe_distance_bytes.argtypes = [C.c_void_p]
        L.swe_distance_copy.restype = C.c_int
        L.swe_distance_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.swe_lpt_partition.restype = None
        L.swe_lpt_partition.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
        L.swe_cost_order.restype = None
        L.swe_cost_order.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        L.swe_capped_linkage.restype = None
        L.swe_capped_linkage.argtypes = [C.c_int, C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
        L.swe_adaptive_matrix.restype = C.c_int
        L.swe_adaptive_matrix.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_float, C.c_int, C.c_char_p, C.c_void_p,
                                          C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.swe_upload_points.restype = C.c_int
        L.swe_upload_points.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.swe_kmer_count.restype = C.c_int64
        L.swe_kmer_count.argtypes = [C.c_int, C.c_int]
        L.swe_kmer_counts.restype = C.c_int
        L.swe_kmer_counts.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int,
                                      C.c_void_p]
        L.swe_kmer_tsv.restype = C.c_int
        L.swe_kmer_tsv.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, TEXT_SINK, C.c_void_p]
        L.frequencies_from_dataset.restype = KmerFrequencies
        L.frequencies_from_dataset.argtypes = [Dataset, C.c_size_t, C.c_int, C.c_int]
        L.write_kmer_base.restype = None
        L.write_kmer_base.argtypes = [C.c_void_p, KmerFrequencies]
        L.free_kmer_frequencies.restype = None
        L.free_kmer_frequencies.argtypes = [KmerFrequencies]
        L.swe_pca_covariance.restype = C.c_int
        L.swe_pca_covariance.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                         C.POINTER(PcaInfo)]
        L.swe_pca_eigen.restype = C.c_int
        L.swe_pca_eigen.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]
        L.swe_pca_eigen_gpu.restype = C.c_int
        L.swe_pca_eigen_gpu.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]
        L.swe_pca_project.restype = C.c_int
        L.swe_pca_project.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int64,
                                      C.c_void_p, C.POINTER(PcaInfo)]
        L.swe_pca.restype = C.c_int
        L.swe_pca.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                              C.POINTER(PcaInfo)]
        _lib = L
    return _lib


def _check(st: int, ctx=None):
    if st != 0:
        msg = lib().swe_last_error(ctx).decode() if ctx else ""
        raise SwgpuError(st, msg)


def split_set_to_lists(s: SplitSet):
    return [[s.clusters[c].members[k] for k in range(s.clusters[c].n_members)]
            for c in range(s.n_clusters)]


class SeqBuffer:
    """Sequences as NUL-terminated C strings in one contiguous host block
    (kept alive with the object): ptrs / lens are the addresses of the
    pointer and length arrays the C calls take."""

    def __init__(self, seqs):
        self.n = len(seqs)
        lens = np.fromiter(map(len, seqs), dtype=np.int64, count=self.n)
        off = np.zeros(self.n + 1, dtype=np.int64)
        np.cumsum(lens + 1, out=off[1:])
        self._blob = b"\0".join(list(seqs) + [b""])  # every sequence followed by its NUL
        base = C.cast(C.c_char_p(self._blob), C.c_void_p).value  # the C calls only read it
        self._ptr = (base + off[:-1]).astype(np.uint64) if self.n else np.zeros(1, dtype=np.uint64)
        self._len = lens.astype(np.uint64) if self.n else np.zeros(1, dtype=np.uint64)
        self.ptrs = self._ptr.ctypes.data
        self.lens = self._len.ctypes.data

    def dataset(self) -> Dataset:
        mx = int(self._len.max()) if self.n else 0
        return Dataset(self._ptr.ctypes.data_as(C.POINTER(C.c_char_p)),
                       self._len.ctypes.data_as(C.POINTER(C.c_size_t)), None, self.n, None, 0, mx)


class Engine:
    """One engine context (one CUDA stream on one device)."""

    def __init__(self, device: int = 0, sat_limit: int = 0, packs_per_block: int = 0, threads: int = 0,
                 inject_timeout: int = 0, threshold_path: int = 0, kmer_batch_kb: int = 0, max_w: int = 0,
                 dbscan_replay: int = 0):
        self.ctx = C.c_void_p()
        opts = Opts(device, sat_limit, packs_per_block, threads, inject_timeout, threshold_path, kmer_batch_kb,
                    max_w, dbscan_replay)
        _check(lib().swe_create(C.byref(self.ctx), C.byref(opts)))
        self.n = 0
        self._buf = None

    def close(self):
        if self.ctx:
            lib().swe_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, seqs):
        self._buf = SeqBuffer(seqs)
        _check(lib().swe_upload(self.ctx, self._buf.ptrs, self._buf.lens, self._buf.n), self.ctx)
        self.n = self._buf.n
        self.set_first = [0, self.n]

    def set_partition(self, part: int, nparts: int):
        """Score only tile group `part` of `nparts` (see swgpu.split_pass)."""
        _check(lib().swe_set_partition(self.ctx, part, nparts), self.ctx)

    def distance_bytes(self) -> int:
        return int(lib().swe_distance_bytes(self.ctx))

    def distance_copy(self, dev_ptr: int, to_engine: bool):
        """Device-to-device copy of the distance storage to / from dev_ptr."""
        _check(lib().swe_distance_copy(self.ctx, C.c_void_p(dev_ptr), int(bool(to_engine))), self.ctx)

    def upload_points(self, values: np.ndarray, metric: int):
        """Points values[dim][point] (float32) with the L1 (metric 1) or L2
        (metric 2) distances of dbscan_L1 / dbscan_L2, computed on upload;
        distances() then returns their float bit patterns."""
        V = np.ascontiguousarray(values, dtype=np.float32)
        if V.ndim != 2:
            raise ValueError("values must be dims x n")
        dims, n = V.shape
        self._pts = V
        ptrs = (C.c_void_p * max(1, dims))(*[V.ctypes.data + k * n * 4 for k in range(dims)])
        _check(lib().swe_upload_points(self.ctx, ptrs, dims, n, metric), self.ctx)
        self._buf = None
        self.n = n
        self.set_first = [0, n]

    def upload_sets(self, sets):
        """Uploads independent sets (a list of sequence lists); pairs are
        scored only inside a set."""
        flat = [q for st in sets for q in st]
        first = np.zeros(len(sets) + 1, dtype=np.int32)
        first[1:] = np.cumsum([len(st) for st in sets])
        self._buf = SeqBuffer(flat)
        _check(lib().swe_upload_sets(self.ctx, self._buf.ptrs, self._buf.lens, self._buf.n, first.ctypes.data,
                                     len(sets)), self.ctx)
        self.n = self._buf.n
        self.set_first = first.tolist()

    def set_count(self) -> int:
        return lib().swe_set_count(self.ctx)

    def set_size(self, set: int) -> int:
        return self.set_first[set + 1] - self.set_first[set]

    def score_all_pairs(self):
        _check(lib().swe_score_all_pairs(self.ctx), self.ctx)

    def distances(self, set: int | None = None) -> np.ndarray:
        if set is None:
            out = np.zeros((self.n, self.n), dtype=np.uint32)
            _check(lib().swe_copy_distances(self.ctx, out.ctypes.data), self.ctx)
        else:
            ns = self.set_size(set)
            out = np.zeros((ns, ns), dtype=np.uint32)
            _check(lib().swe_copy_set_distances(self.ctx, set, out.ctypes.data), self.ctx)
        return out

    def partition_bytes(self, part: int) -> int:
        """Bytes of group `part`'s payload in the split pass's exchange."""
        b = lib().swe_partition_bytes(self.ctx, part)
        if b < 0:
            raise SwgpuError(1, "no such group")
        return int(b)

    def partition_pack(self, dev_ptr: int):
        _check(lib().swe_partition_pack(self.ctx, C.c_void_p(dev_ptr)), self.ctx)

    def partition_unpack(self, part: int, dev_ptr: int, offset: int, nbytes: int):
        _check(lib().swe_partition_unpack(self.ctx, part, C.c_void_p(dev_ptr), offset, nbytes), self.ctx)

    def autotune(self, seqs, cache_path: str | None = None, force: bool = False) -> dict:
        """Times the 16x2 kernel's tile plans on a length-stratified sample of
        `seqs` and sets the fastest on this engine (see swe_autotune)."""
        buf = SeqBuffer(seqs)
        res = TuneResult()
        _check(lib().swe_autotune(self.ctx, buf.ptrs, buf.lens, len(seqs),
                                  cache_path.encode() if cache_path else None, 1 if force else 0,
                                  C.byref(res)), self.ctx)
        return res.as_dict()

    def rows(self, row0: int, row1: int, set: int = 0) -> np.ndarray:
        """Rows [row0, row1) of one set's distance matrix (original order)."""
        ns = self.set_size(set)
        out = np.zeros((row1 - row0, ns), dtype=np.uint32)
        _check(lib().swe_copy_set_rows(self.ctx, set, row0, row1, out.ctypes.data), self.ctx)
        return out

    def neighbors(self, eps: float, set: int | None = None):
        rp, cols = C.c_void_p(), C.c_void_p()
        if set is None:
            _check(lib().swe_neighbors(self.ctx, C.c_float(eps), C.byref(rp), C.byref(cols)), self.ctx)
            n = self.n
        else:
            _check(lib().swe_neighbors_set(self.ctx, set, C.c_float(eps), C.byref(rp), C.byref(cols)), self.ctx)
            n = self.set_size(set)
        row_ptr = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_int64)), shape=(n + 1,)).copy()
        E = int(row_ptr[-1])
        c = (np.ctypeslib.as_array(C.cast(cols, C.POINTER(C.c_int32)), shape=(max(E, 1),))[:E].copy()
             if E else np.zeros(0, dtype=np.int32))
        lib().swe_free(rp)
        lib().swe_free(cols)
        return row_ptr, c

    def dbscan(self, eps: float, minpts: int, set: int | None = None, lists: bool = True):
        """Clusters as member lists, or their number with lists=False."""
        s = SplitSet()
        if set is None:
            _check(lib().swe_dbscan(self.ctx, C.c_float(eps), minpts, C.byref(s)), self.ctx)
        else:
            _check(lib().swe_dbscan_set(self.ctx, set, C.c_float(eps), minpts, C.byref(s)), self.ctx)
        out = split_set_to_lists(s) if lists else s.n_clusters
        lib().free_split_set_and_associated_clusters(s)
        return out

    def adaptive(self, eps_start: float, eps_inc: float, minpts: int, prefix: str | None = None,
                 log_path: str | None = None, set: int | None = None, layers: bool = True):
        """Runs the sweep; returns (log text, kept split sets as lists), or
        (log text, number of kept layers) with layers=False (the layers stay
        in the library and are freed there)."""
        libc = C.CDLL(None)
        libc.fopen.restype = C.c_void_p
        libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
        libc.fclose.argtypes = [C.c_void_p]
        import tempfile
        tmp = None
        if log_path is None:
            fd, tmp = tempfile.mkstemp(prefix="swgpu_log_")
            os.close(fd)
            log_path = tmp
        f = libc.fopen(log_path.encode(), b"w")
        sets = C.POINTER(SplitSet)()
        nsets = C.c_int()
        pre = prefix.encode() if prefix else None
        out = C.byref(sets) if layers else None
        if set is None:
            st = lib().swe_adaptive(self.ctx, C.c_float(eps_start), C.c_float(eps_inc), minpts, pre, f,
                                    out, C.byref(nsets))
        else:
            st = lib().swe_adaptive_set(self.ctx, set, C.c_float(eps_start), C.c_float(eps_inc), minpts, pre, f,
                                        out, C.byref(nsets))
        libc.fclose(f)
        text = Path(log_path).read_text()
        if tmp:
            os.unlink(tmp)
        _check(st, self.ctx)
        if not layers:
            return text, nsets.value
        kept = [split_set_to_lists(sets[k]) for k in range(nsets.value)]
        for k in range(nsets.value):
            lib().free_split_set_and_associated_clusters(sets[k])
        lib().swe_free(sets)
        return text, kept

    def adaptive_sets(self, eps_start: float, eps_inc: float, minpts: int, max_steps: int = 0,
                      prefix: str | None = None, layers: bool = True):
        """Sweeps of every uploaded set at once; one dict per set with its
        status, truncated flag, steps, log text, kept layers (their number
        with layers=False) and done_ms."""
        S = self.set_count()
        res = (SweepResult * max(S, 1))()
        _check(lib().swe_adaptive_sets(self.ctx, C.c_float(eps_start), C.c_float(eps_inc), minpts, max_steps,
                                       prefix.encode() if prefix else None, res), self.ctx)
        out = []
        for k in range(S):
            r = res[k]
            out.append({"status": r.status, "truncated": bool(r.truncated), "steps": r.steps,
                        "log": C.string_at(r.log).decode("latin-1") if r.log else "",
                        "layers": ([split_set_to_lists(r.layers[i]) for i in range(r.n_layers)] if layers
                                   else r.n_layers),
                        "done_ms": r.done_ms})
        lib().swe_free_sweep_results(res, S)
        return out

    # ---------------------------------------------------------------- fasta2kmer
    @staticmethod
    def _row_ptrs(table: np.ndarray):
        n, nk = table.shape
        base = table.ctypes.data
        return (C.c_void_p * max(1, n))(*[base + i * nk * 2 for i in range(n)])

    def kmer_counts(self, seqs, k: int, protein: bool = False) -> np.ndarray:
        """k-mer frequency table of frequencies_from_dataset (kmers.c:292-371)
        over len(s) bytes of each sequence: int16 array (n, 4^k or 20^k)."""
        nk = lib().swe_kmer_count(k, int(bool(protein)))
        if nk == 0:
            raise SwgpuError(1, "k-mer length out of range")
        buf = SeqBuffer(seqs)
        n = len(seqs)
        out = np.zeros((n, nk), dtype=np.int16)
        lens = (C.c_int64 * max(1, n))(*[len(s) for s in seqs])
        _check(lib().swe_kmer_counts(self.ctx, buf.ptrs, lens, n, k, int(bool(protein)), self._row_ptrs(out)),
               self.ctx)
        return out

    def kmer_tsv(self, table: np.ndarray) -> bytes:
        """The text write_kmer_base (kmers.c:373-385) prints for a table."""
        t = np.ascontiguousarray(table, dtype=np.int16)
        chunks = []

        @TEXT_SINK
        def sink(data, size, _user):
            chunks.append(C.string_at(data, size))
            return 0

        _check(lib().swe_kmer_tsv(self.ctx, self._row_ptrs(t), t.shape[0], t.shape[1], sink, None), self.ctx)
        return b"".join(chunks)

    # ---------------------------------------------------------------- kmer2pca
    def pca_covariance(self, table) -> tuple[np.ndarray, dict]:
        """means_from_data + feature_covariance_matrix (kmer2pca.c:286-481) of
        a (samples, features) table on the GPU: the covariance matrix and the
        call's swe_pca_info.  The table stays on the GPU for pca_project(None, ...)."""
        X = np.ascontiguousarray(table, dtype=np.float64)
        n, nf = X.shape
        cov = np.zeros((nf, nf))
        info = PcaInfo()
        _check(lib().swe_pca_covariance(self.ctx, X.ctypes.data, n, nf, cov.ctypes.data, C.byref(info)), self.ctx)
        self._pca_rows = n
        return cov, info.as_dict()

    def pca_eigen(self, cov, n_vectors: int) -> tuple[np.ndarray, np.ndarray]:
        """swgpu.pca_eigen with the reduction and the bisection on the GPU
        (swe_pca_eigen_gpu)."""
        A = np.ascontiguousarray(cov, dtype=np.float64)
        n = A.shape[0]
        w = np.zeros(n)
        V = np.zeros((max(n_vectors, 1), n))
        _check(lib().swe_pca_eigen_gpu(self.ctx, A.ctypes.data, n, n_vectors, w.ctypes.data, V.ctypes.data),
               self.ctx)
        return w, V[:n_vectors]

    def pca_project(self, table, vectors) -> np.ndarray:
        """obtain_projections (kmer2pca.c:141-211): (samples, len(vectors)) sums
        of table row x vector in the order of the features; table None projects
        the table of the last pca_covariance / pca call."""
        V = np.ascontiguousarray(vectors, dtype=np.float64)
        d, nf = V.shape
        if table is None:
            ptr, n = None, getattr(self, "_pca_rows", 0)
        else:
            X = np.ascontiguousarray(table, dtype=np.float64)
            ptr, n = X.ctypes.data, X.shape[0]
        out = np.zeros((n, d))
        _check(lib().swe_pca_project(self.ctx, ptr, n, nf, V.ctypes.data, d, out.ctypes.data, None), self.ctx)
        return out

    def pca(self, table, dimensions: int) -> tuple[np.ndarray, np.ndarray, dict]:
        """kmer2pca after its file is read (kmer2pca.c:540-586): every
        eigenvalue (ascending), the projections onto the `dimensions` leading
        eigenvectors, and the call's swe_pca_info."""
        X = np.ascontiguousarray(table, dtype=np.float64)
        n, nf = X.shape
        w = np.zeros(nf)
        P = np.zeros((n, dimensions))
        info = PcaInfo()
        _check(lib().swe_pca(self.ctx, X.ctypes.data, n, nf, dimensions, w.ctypes.data, P.ctypes.data,
                             C.byref(info)), self.ctx)
        self._pca_rows = n
        return w, P, info.as_dict()

    # ---------------------------------------------------------------- prefilter
    def kmer_features(self, k: int = 5) -> np.ndarray:
        out = np.zeros((self.n, 4 ** k), dtype=np.float32)
        _check(lib().swe_kmer_features(self.ctx, k, out.ctypes.data), self.ctx)
        return out

    def prefilter_init(self, seed: int = 0):
        _check(lib().swe_prefilter_init(self.ctx, seed), self.ctx)

    def prefilter_params(self, set_to: np.ndarray | None = None) -> np.ndarray:
        n = lib().swe_prefilter_param_count()
        out = np.zeros(n, dtype=np.float32)
        src = None
        if set_to is not None:
            src = np.ascontiguousarray(set_to, dtype=np.float32)
            assert src.size == n
        _check(lib().swe_prefilter_params(self.ctx, out.ctypes.data, src.ctypes.data if src is not None else None),
               self.ctx)
        return out if set_to is None else src.copy()

    @staticmethod
    def _pairs(a, b, d=None):
        a = np.ascontiguousarray(a, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.int32)
        d = None if d is None else np.ascontiguousarray(d, dtype=np.uint32)
        return a, b, d

    def prefilter_loss_grad(self, a, b, dist):
        a, b, d = self._pairs(a, b, dist)
        loss = C.c_float()
        grad = np.zeros(lib().swe_prefilter_param_count(), dtype=np.float32)
        _check(lib().swe_prefilter_loss_grad(self.ctx, a.ctypes.data, b.ctypes.data, d.ctypes.data, len(a),
                                             C.byref(loss), grad.ctypes.data), self.ctx)
        return loss.value, grad

    def prefilter_train(self, a, b, dist, epochs: int, batch_pairs: int = 4096, lr: float = 1e-3, seed: int = 0,
                        weight_decay: float = 0.0, over_eps: float = 0.0, over_weight: float = 1.0):
        a, b, d = self._pairs(a, b, dist)
        losses = np.zeros(max(epochs, 1), dtype=np.float32)
        _check(lib().swe_prefilter_train(self.ctx, a.ctypes.data, b.ctypes.data, d.ctypes.data, len(a), epochs,
                                         batch_pairs, C.c_float(lr), C.c_float(weight_decay), seed,
                                         C.c_float(over_eps), C.c_float(over_weight), losses.ctypes.data),
               self.ctx)
        return losses[:epochs]

    def prefilter_embed(self) -> np.ndarray:
        out = np.zeros((self.n, 128), dtype=np.float32)
        _check(lib().swe_prefilter_embed(self.ctx, out.ctypes.data), self.ctx)
        return out

    def prefilter_pair_dist(self, a, b) -> np.ndarray:
        a, b, _ = self._pairs(a, b)
        out = np.zeros(len(a), dtype=np.float32)
        _check(lib().swe_prefilter_pair_dist(self.ctx, a.ctypes.data, b.ctypes.data, len(a), out.ctypes.data),
               self.ctx)
        return out

    def prefilter_set_embeddings(self, emb: np.ndarray):
        emb = np.ascontiguousarray(emb, dtype=np.float32)
        assert emb.shape == (self.n, 128)
        _check(lib().swe_prefilter_set_embeddings(self.ctx, emb.ctypes.data), self.ctx)

    def score_prefiltered(self, eps: float, margins, use_emb: bool = True) -> dict:
        """Prefiltered score pass; margins: a float or [(upper_len, margin), ...]."""
        st = PrefilterStats()
        mt = Margins.of(margins)
        _check(lib().swe_score_prefiltered(self.ctx, C.c_float(eps), C.byref(mt), int(use_emb), C.byref(st)),
               self.ctx)
        return st.as_dict()

    def dbscan_bitmaps_device(self, instances, minpts: int):
        """Device replays of many DBSCAN instances in one launch; instances is
        a list of (bits [n, wpr] uint64, counts [n] int32).  Returns each
        instance's clusters as lists of member indices."""
        k = len(instances)
        ns = np.array([len(c) for _, c in instances], dtype=np.int32)
        boff = np.zeros(k, dtype=np.int64)
        coff = np.zeros(k, dtype=np.int64)
        bw = cw = 0
        for i, (b, c) in enumerate(instances):
            boff[i], coff[i] = bw, cw
            bw += int(np.asarray(b).size)
            cw += len(c)
        bits = np.concatenate([np.asarray(b, dtype=np.uint64).ravel() for b, _ in instances] + [np.zeros(1, np.uint64)])
        counts = np.concatenate([np.asarray(c, dtype=np.int32) for _, c in instances] + [np.zeros(1, np.int32)])
        out = (SplitSet * max(k, 1))()
        _check(lib().swe_dbscan_bitmaps_device(self.ctx, k, ns.ctypes.data, bits.ctypes.data, boff.ctypes.data, bw,
                                               counts.ctypes.data, coff.ctypes.data, cw, minpts, out), self.ctx)
        res = []
        for i in range(k):
            res.append(split_set_to_lists(out[i]))
            lib().free_split_set_and_associated_clusters(out[i])
        return res

    def one_to_many(self, q: bytes, qlen: int | None = None) -> np.ndarray:
        qlen = len(q) if qlen is None else qlen
        buf = C.create_string_buffer(bytes(q), max(len(q), qlen) + 1)
        out = np.zeros(self.n, dtype=np.uint32)
        _check(lib().swe_score_one_to_many(self.ctx, buf, qlen, out.ctypes.data), self.ctx)
        return out

    def score_pairs(self, a, b) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.int32)
        out = np.zeros(len(a), dtype=np.uint32)
        _check(lib().swe_score_pairs(self.ctx, a.ctypes.data, b.ctypes.data, len(a), out.ctypes.data),
               self.ctx)
        return out

    def timer_start(self):
        _check(lib().swe_timer_start(self.ctx), self.ctx)

    def timer_stop(self) -> float:
        ms = C.c_double()
        _check(lib().swe_timer_stop(self.ctx, C.byref(ms)), self.ctx)
        return ms.value

    def stats(self) -> dict:
        s = Stats()
        _check(lib().swe_get_stats(self.ctx, C.byref(s)))
        return s.as_dict()


def dbscan_from_matrix(D: np.ndarray, eps: float, minpts: int):
    """DBSCAN replay (host) on neighbourhoods thresholded from a distance matrix
    the caller already holds: (float)D[i][k] <= eps."""
    D = np.asarray(D)
    n = D.shape[0]
    nb = D.astype(np.float32) <= np.float32(eps)
    wpr = (n + 63) // 64
    padded = np.zeros((n, wpr * 64), dtype=bool)
    padded[:, :n] = nb
    bits = np.packbits(padded.reshape(n, wpr, 64)[:, :, ::-1], axis=2).reshape(n, wpr * 8)
    words = np.ascontiguousarray(bits).view(">u8").astype(np.uint64).reshape(n, wpr)
    counts = np.ascontiguousarray(nb.sum(axis=1), dtype=np.int32)
    s = SplitSet()
    _check(lib().swe_dbscan_bitmap(n, words.ctypes.data, wpr, counts.ctypes.data, minpts, C.byref(s)))
    out = split_set_to_lists(s)
    lib().free_split_set_and_associated_clusters(s)
    return out


def adaptive_from_matrix(D: np.ndarray, eps_start: float, eps_inc: float, minpts: int, speculate: bool = True,
                         batch: int = 8, prefix: str | None = None):
    """The adaptive sweep on the host over a distance matrix the caller holds
    (swe_adaptive_matrix); returns (log text, kept split sets as lists)."""
    import tempfile
    D = np.ascontiguousarray(D, dtype=np.uint32)
    n = D.shape[0]
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    fd, tmp = tempfile.mkstemp(prefix="swgpu_log_")
    os.close(fd)
    f = libc.fopen(tmp.encode(), b"w")
    sets = C.POINTER(SplitSet)()
    nsets = C.c_int()
    st = lib().swe_adaptive_matrix(n, D.ctypes.data, C.c_float(eps_start), C.c_float(eps_inc), minpts,
                                   prefix.encode() if prefix else None, f, int(speculate), batch, C.byref(sets),
                                   C.byref(nsets))
    libc.fclose(f)
    text = Path(tmp).read_text()
    os.unlink(tmp)
    if st != 0:
        return text, None
    kept = [split_set_to_lists(sets[k]) for k in range(nsets.value)]
    for k in range(nsets.value):
        lib().free_split_set_and_associated_clusters(sets[k])
    lib().swe_free(sets)
    return text, kept


def pca_eigen(cov, n_vectors: int) -> tuple[np.ndarray, np.ndarray]:
    """eigen_from_corr (kmer2pca.c:107-138) on the host: every eigenvalue of
    the symmetric matrix, ascending, and the unit eigenvectors of the
    n_vectors largest ones, largest first (rows; sign: largest-magnitude entry
    positive)."""
    A = np.ascontiguousarray(cov, dtype=np.float64)
    n = A.shape[0]
    w = np.zeros(n)
    V = np.zeros((max(n_vectors, 1), n))
    _check(lib().swe_pca_eigen(A.ctypes.data, n, n_vectors, w.ctypes.data, V.ctypes.data))
    return w, V[:n_vectors]


def capped_linkage(n: int, pairs, cap: int) -> np.ndarray:
    """Group label (the group's smallest index) of each of n items after
    single linkage over the (a, b) rows of `pairs` in order, no group larger
    than `cap` - the grouping of the prefiltered pass."""
    p = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    label = np.zeros(max(1, n), dtype=np.int32)
    lib().swe_capped_linkage(n, p.ctypes.data, len(p), cap, label.ctypes.data)
    return label[:n]


def cost_order(cost) -> np.ndarray:
    """Indices of `cost` by descending cost, ties in index order: the order of
    the score pass's tile list."""
    c = np.ascontiguousarray(cost, dtype=np.float64)
    order = np.zeros(max(1, len(c)), dtype=np.int32)
    lib().swe_cost_order(c.ctypes.data, len(c), order.ctypes.data)
    return order[:len(c)]


def lpt_partition(cost, nparts: int) -> np.ndarray:
    """Group of each tile (costs in descending order) as swe_set_partition assigns them."""
    c = np.ascontiguousarray(cost, dtype=np.float64)
    owner = np.zeros(max(1, len(c)), dtype=np.int32)
    lib().swe_lpt_partition(c.ctypes.data, len(c), nparts, owner.ctypes.data)
    return owner[:len(c)]


def measure_mix_peak(device: int = 0):
    """(DP cells/s, lane instructions/s) of the 16x2 per-cell instruction mix."""
    c, i = C.c_double(), C.c_double()
    _check(lib().swe_measure_mix_peak(device, C.byref(c), C.byref(i)))
    return c.value, i.value


def score(a: bytes, b: bytes, la: int | None = None, lb: int | None = None) -> int:
    """The drop-in score() (one pair on the GPU)."""
    la = len(a) if la is None else la
    lb = len(b) if lb is None else lb
    ab = C.create_string_buffer(bytes(a), max(len(a), la) + 1)
    bb = C.create_string_buffer(bytes(b), max(len(b), lb) + 1)
    d = lib().score(ab, bb, la, lb, None)
    st = lib().swgpu_last_dropin_status()
    if d == 0xFFFFFFFF and st:
        raise SwgpuError(st, "score failed")
    return d
