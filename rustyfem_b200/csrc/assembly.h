// Assembly of the stiffness matrix K on the GPU: the tangent branch of
// `internal` (src/fem/assembly.rs:315-420) for a symmetric system matrix
// without constraints, into the values of the solver's lower CSC pattern
// (src/sparse.rs:256-275, internal numbering).
//
// The reference computes the element matrices in parallel and then adds them
// one element after another through SystemMatrix::add (a binary search into
// the column, src/sparse.rs:47-51), K_ab += ½(ke[a,b] + ke[b,a]) for every
// pair of element DOFs with equations ia >= ib. Here the pairs are mapped once
// (prepare): each lower entry gets the list of (element, a, b) that reach it,
// sorted by element and then by (a, b), which is the reference's order of
// additions into that entry. An assembly is then one thread per entry summing
// its list from zero in that order: the same sums, bit for bit, with no atomics.
//
//   k_asm_count / k_asm_fill   one thread per (element, a, b): the entry by binary
//                              search, a count per entry, then the keys placed
//                              (prefix sum of the counts between them)
//   sort_rows_u64              each entry's keys sorted (element, a, b)
//   k_asm_gather               one thread per entry: Σ ½(ke[a,b] + ke[b,a])
//   k_ke_hex8                  one CTA per C3D8 element: its 24×24 matrix
//                              (src/elements/continuum3d.rs:39-131)
// The file is compiled without multiply-add contraction.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace rfg {

class Assembler {
   public:
    // n equations; colptr/rowidx: the lower CSC pattern (host); nelem elements of nd DOFs
    // with equations edof[e·nd + a] (host; -1 = none). Throws CudaError if an element pair
    // is not in the pattern (message names the entry).
    Assembler(int64_t n, const int64_t* colptr, const int64_t* rowidx, int64_t nelem, int64_t nd, const int64_t* edof,
              cudaStream_t st);
    ~Assembler();
    Assembler(const Assembler&) = delete;
    Assembler& operator=(const Assembler&) = delete;

    // Writes K into val (device, nnz values) from element matrices ke (nelem·nd·nd,
    // row-major per element) in host or device memory.
    void assemble(const double* ke, bool ke_on_device, double* val);
    // C3D8 elements: K_e of each element on the device, then assembled into val. conn:
    // nelem × 8 node ids, xyz: nn × 3, emod: E per element (host). Returns -1, or the
    // first element whose Jacobian is not positive at an integration point.
    int64_t hex8(int64_t nn, const double* xyz, const int64_t* conn, const double* emod, double nu, double* val);

    int64_t nnz() const { return nnz_; }
    int64_t contributions() const { return ncontrib_; }
    // device time of the last element kernel and of the last gather (ms)
    double element_ms() const { return element_ms_; }
    double gather_ms() const { return gather_ms_; }

   private:
    void ensure_ke();
    int64_t n_, nnz_, nelem_, nd_, ncontrib_ = 0;
    cudaStream_t st_;
    int64_t* d_start_ = nullptr;    // nnz + 1: first key of each entry
    uint64_t* d_key_ = nullptr;     // (e·nd + a)·nd + b per contribution
    double* d_ke_ = nullptr;        // element matrices (device copy or kernel output)
    double* d_xyz_ = nullptr;
    int64_t* d_conn_ = nullptr;
    double* d_emod_ = nullptr;
    int64_t nn_cap_ = 0;
    long long* d_bad_ = nullptr;
    cudaEvent_t ev_[3] = {nullptr, nullptr, nullptr};
    double element_ms_ = 0.0, gather_ms_ = 0.0;
};

}  // namespace rfg
