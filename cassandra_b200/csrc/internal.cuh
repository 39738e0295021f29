// Internal declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"
#include "patterns.h"

namespace cas {

struct DevicePatterns {
    Instance* instances = nullptr;
    uint32_t* tables = nullptr;
    int k = 0;
    int64_t cols = 0;
};

// Positions still arriving on another stream, in row chunks: chunk i (rows
// [row_end[i-1], row_end[i]), row_end[-1] = 0) is on the device once
// ready[i] has completed.  A build given this launches the indexing of each
// chunk behind its event, so that the copy of the next chunk overlaps it.
struct PositionChunks {
    int n = 0;
    const int64_t* row_end = nullptr;
    const cudaEvent_t* ready = nullptr;
};

cas_status require_device();
cas_status patterns_on_device(const cas_patterns* p, const DevicePatterns** out);
const PatternSet& pattern_set(const cas_patterns* p);
cas_status launch_index(const DevicePatterns& dp, const uint64_t* d_pos, int64_t n, uint32_t* d_out,
                        cudaStream_t stream);
// Several solvers to tolerance at once, each on its own stream; per-solver
// statuses in sts, reports in reps (may be null).  Returns the first failed
// CUDA call's status (solver.cu).
cas_status solvers_run_all(cas_solver* const* svs, int n, cas_solve_report* reps, cas_status* sts);
// cas_csr_from_positions_layout with positions that may still be arriving
// (chunks may be null: all on the device) (csr.cu).
cas_status csr_from_positions(const cas_patterns* p, const uint64_t* d_positions, int64_t rows, int layouts,
                              cudaStream_t s, cas_csr** out, const PositionChunks* chunks);

// Entries of one A'y work unit: a column's row list is cut into units of at
// most kUnit entries, one warp each.
constexpr int kUnit = 2048;

// Device-side arrays that the products need.
struct CsrView {
    int64_t rows = 0, cols = 0;
    int k = 0;
    const uint32_t* idx = nullptr;       // rows * k, row-major
    const int64_t* col_ptr = nullptr;    // cols + 1
    const uint32_t* row_idx = nullptr;   // nnz, sorted by (col, row)
    int64_t units = 0;
    const int32_t* unit_col = nullptr;   // units
    const uint32_t* unit_ptr = nullptr;  // cols + 1: first unit of each column
    const uint64_t* diag_int = nullptr;  // cols: diag(A'A) as integers
};

}  // namespace cas

namespace cas {
struct FastLayout;
}

struct cas_csr {
    int device = -1;
    int layouts = 0;                 // CAS_LAYOUT_* bits present
    cas::FastLayout* fast = nullptr;  // blocked layout (fast.cuh), or null
    int64_t rows = 0, cols = 0;
    int k = 0;
    uint32_t* idx = nullptr;
    int64_t* col_ptr = nullptr;
    uint32_t* row_idx = nullptr;
    int64_t units = 0;
    int32_t* unit_col = nullptr;
    uint32_t* unit_ptr = nullptr;
    uint64_t* diag_int = nullptr;
    double* unit_partial = nullptr;  // scratch of A'y: one double per unit
    cas::CsrView view() const
    {
        cas::CsrView v;
        v.rows = rows;
        v.cols = cols;
        v.k = k;
        v.idx = idx;
        v.col_ptr = col_ptr;
        v.row_idx = row_idx;
        v.units = units;
        v.unit_col = unit_col;
        v.unit_ptr = unit_ptr;
        v.diag_int = diag_int;
        return v;
    }
};

namespace cas {

// Product kernels (csr.cu), usable by the solver.
template <typename T>
cas_status spmv(const CsrView& a, const T* x, T* y, cudaStream_t s);
template <typename T>
cas_status spmv_t(const CsrView& a, const T* y, double* unit_partial, T* x, cudaStream_t s);
template <typename T>
cas_status jacobi(const CsrView& a, T* out, cudaStream_t s);

}  // namespace cas
