// Host symbolic stage of the multifrontal LDLᵀ: geometric nested dissection on
// the node graph, postorder numbering of the equations, front patterns, flop
// estimate and the lower-triangle CSC pattern. It follows the reference's
// analysis (src/sparse.rs:78-275) so that the tree, the front list and the
// equation numbering are those of the reference solver.
#pragma once

#include <cstddef>
#include <cstdint>
#include <new>
#include <utility>
#include <vector>

namespace rfg {

// Host blocks of at least HOST_BLOCK_MIN bytes come from a process-wide cache of freed
// blocks (hostmem.cpp): the large scratch arrays of one factorization call reuse the pages
// of the previous call instead of faulting in fresh ones. host_release_cached() frees the
// cached blocks (rfg_release_cached_memory).
constexpr size_t HOST_BLOCK_MIN = (size_t)1 << 20;
void* host_block_alloc(size_t bytes);
void host_block_free(void* p);
void host_release_cached();

// Allocator that leaves trivially constructible elements uninitialised on resize():
// for large host arrays that are overwritten entirely right after. Large blocks come
// from the host block cache.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    T* allocate(size_t n) {
        if (n * sizeof(T) >= HOST_BLOCK_MIN) return static_cast<T*>(host_block_alloc(n * sizeof(T)));
        return std::allocator<T>::allocate(n);
    }
    void deallocate(T* p, size_t n) {
        if (n * sizeof(T) >= HOST_BLOCK_MIN)
            host_block_free(p);
        else
            std::allocator<T>::deallocate(p, n);
    }
    template <typename U>
    void construct(U* p) noexcept {
        ::new ((void*)p) U;
    }
    template <typename U, typename... Args>
    void construct(U* p, Args&&... args) {
        ::new ((void*)p) U(std::forward<Args>(args)...);
    }
};
template <typename T>
using HostVec = std::vector<T, NoInitAlloc<T>>;
using SegVec = HostVec<int64_t>;

struct Graph {
    int64_t nn = 0;
    const double* coords = nullptr;  // 3 per node
    std::vector<int64_t> adj_ptr;    // nn+1
    SegVec adj_idx;                  // neighbours, self excluded
    std::vector<int64_t> ndof;       // DOFs per node
};

struct SymFront {
    int64_t start = 0;               // first pivot equation
    int64_t k = 0;                   // pivots
    int64_t rows_off = 0;            // offset of the front's later rows in Symbolic::rows
    int64_t u = 0;                   // number of later rows
    int64_t parent = -1;
    int64_t child_off = 0, nchild = 0;  // children in Symbolic::children
    double work = 0.0;               // flops of the whole subtree
};

struct Symbolic {
    int64_t n = 0;                   // equations
    std::vector<int64_t> first_dof;  // per node
    std::vector<SymFront> fronts;    // in postorder (children before parents)
    SegVec rows;                     // concatenated sorted later rows of the fronts
    std::vector<int64_t> children;   // concatenated child indices
    std::vector<int64_t> roots;
    std::vector<int64_t> front_nodes_off, front_nodes;  // nodes of each front in pivot order

    double work() const;             // src/sparse.rs:236-238
    int64_t factor_size() const;     // src/sparse.rs:241-243
    void largest_front(int64_t* k, int64_t* u) const;  // src/sparse.rs:251-253
};

// src/sparse.rs:167-232 (leaf_max: 48 for the engine, 16 for the C interface)
Symbolic analyse(const Graph& g, int64_t leaf_max);

// src/sparse.rs:256-275: CSC of the lower triangle in the internal numbering
void lower_pattern(const Symbolic& s, const Graph& g, std::vector<int64_t>& colptr, std::vector<int64_t>& rowidx);

}  // namespace rfg
