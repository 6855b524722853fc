// Minimal stand-ins for the XAMG types that the reference's loop files use,
// so that those files compile unchanged, where they lie, into a CPU library
// that checks the oracle (test infrastructure only; never part of the product).
//
// The reference's loop bodies (src/blas/detail/blas.inl, blas_ext.inl,
// src/blas2/detail/csr_matvec.inl, csr_gs.inl, dense_matvec.inl) touch their
// operands through a small surface of vector::vector and
// matrix::csr_matrix / dense_matrix: data pointers (get_aligned_ptr), the row
// range of the calling core (get_core_range), a handful of state flags and the
// sharing mode.  Everything here models ONE process with ONE core: the core's
// range is the whole vector and every offset is zero, which is the reference's
// single-process configuration.  The MPI, shared-memory, logging and
// performance-counter hooks the files name are inert.
//
// Each translation unit of a library is compiled with XAMG defined to a name
// of its own (build_ref_loops.py), so that the reference's inline templates
// instantiated under different floating-point flags cannot be merged by the
// linker; units talk to each other only through the C entry points.
//
// Member names and enumerators follow the reference's headers
// (src/primitives/vector/vector.h:45-62, 221; src/xamg_types.h:90-98;
// src/primitives/matrix/csr_matrix.h:47-120) because the included loop files
// refer to them by name; the classes themselves hold no more than a pointer
// and the flags.
#pragma once

#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <typeinfo>
#include <vector>

#include "xamg_macros.h"  // the reference's own vectorisation / restrict macros
#include "misc/rand.h"     // the reference's pseudo-random stream (xorshift32 + LCG)

typedef float float32_t;
typedef double float64_t;
#define XAMG_ALIGN_SIZE 64
#define XAMG_STACK_ALIGNMENT_PREFIX alignas(XAMG_ALIGN_SIZE)
// the constant-vector cache's definitions live in the reference's own
// library object; its loop files skip them under this macro
#define XAMG_SEPARATE_OBJECT

// Process identity (global, as in the reference): one process that is master
// of its node and NUMA domain.
struct ID {
    int gl_proc = 0;
    int gl_nprocs = 1;
    int nd_numa = 0;
    bool master_process() const { return true; }
    bool node_master_process() const { return true; }
    bool numa_master_process() const { return true; }
};

namespace XAMG {

namespace mem {
enum allocation { LOCAL, SHARED, DISTRIBUTED };
enum sharing { NODE, NUMA, NUMA_NODE, CORE };
}  // namespace mem

namespace segment {
enum hierarchy { NODE, NUMA, CORE };
}  // namespace segment

enum multigrid_cycle { V_cycle = 0, F_cycle = 1, W_cycle = 2 };  // xamg_types.h:84

// Performance counters: counted by the reference, ignored here.
struct perf_info {
    void mem_read(int) {}
    void mem_write(int) {}
    void flop(int) {}
    void allreduce(int) {}
    void start() {}
    void stop() {}
};

// The log stream: discards what the reference prints.
enum out_modifier { DBG, ALLRANKS };
struct null_stream {
    template <typename T> const null_stream &operator<<(const T &) const { return *this; }
};
static const null_stream out = {};

namespace mpi {
enum scope { INTRA_NUMA, INTRA_NODE, CROSS_NUMA, CROSS_NODE, GLOBAL };
inline void barrier(scope) {}
// one process: the allreduce of a local value is the value itself
template <typename T> inline void allreduce_sum(const T *in, T *out, int n) {
    for (int i = 0; i < n; ++i) out[i] = in[i];
}
template <typename T> inline void allreduce_bxor(const T *in, T *out, int n) {
    for (int i = 0; i < n; ++i) out[i] = in[i];
}
}  // namespace mpi

namespace vector {

// A block vector of `size` rows and `nv` columns, row-major (x[i*nv + k]),
// viewing caller-owned memory.
struct vector {
    enum vector_status { unallocated, allocated, nonempty, uninitialized, initialized };

    mem::sharing sharing_mode = mem::NUMA_NODE;
    size_t type_hash = typeid(void).hash_code();
    bool if_allocated = false;
    bool if_empty = true;
    bool if_initialized = false;
    bool if_zero = true;
    uint64_t size = 0;
    uint64_t ext_offset = 0;
    uint16_t nv = 0;
    void *ptr = nullptr;
    std::vector<double> own;  // storage for the small vectors the wrappers allocate

    vector() = default;
    explicit vector(mem::sharing m) : sharing_mode(m) {}
    explicit vector(mem::allocation) {}
    template <typename P> void set_part(const P &) {}
    // a copy of a vector that owns its storage views its own copy of it
    vector(const vector &o) { *this = o; }
    vector &operator=(const vector &o) {
        sharing_mode = o.sharing_mode; type_hash = o.type_hash; if_allocated = o.if_allocated;
        if_empty = o.if_empty; if_initialized = o.if_initialized; if_zero = o.if_zero; size = o.size;
        ext_offset = o.ext_offset; nv = o.nv; own = o.own;
        ptr = o.own.empty() ? o.ptr : (void *)own.data();
        return *this;
    }

    template <typename T> void view(T *p, uint64_t n, uint16_t w, bool zero = false) {
        ptr = (void *)p;
        size = n;
        nv = w;
        type_hash = typeid(T).hash_code();
        if_allocated = true;
        if_empty = (n == 0);
        if_initialized = true;
        if_zero = zero;
    }
    template <typename T> T *alloc_and_get_aligned_ptr(uint64_t n, uint16_t w) {
        own.assign((n * w * sizeof(T) + sizeof(double) - 1) / sizeof(double) + 1, 0.0);
        view<T>((T *)own.data(), n, w, true);
        if_initialized = false;
        return (T *)ptr;
    }
    template <typename T> void alloc(uint64_t n, uint16_t w) { alloc_and_get_aligned_ptr<T>(n, w); }
    template <typename T> T *get_aligned_ptr(int = -1) const { return (T *)ptr; }
    template <typename T> void get_core_range(uint64_t &core_size, uint64_t &core_offset) const {
        core_size = size;
        core_offset = 0;
    }
    // row range of a compressed (row-indexed) block: not used with one core
    template <typename I, typename T>
    void get_core_range(uint64_t &core_size, uint64_t &core_offset, const vector &) const {
        core_size = size;
        core_offset = 0;
    }
    uint64_t global_numa_offset() const { return 0; }
    uint64_t numa_offset() const { return 0; }
    uint64_t intra_numa_offset() const { return 0; }
    void check(vector_status) const {}
};

struct indx_vector : vector {
    uint64_t r1 = 0, r2 = 0;
};

}  // namespace vector

namespace matrix {

// CSR block: row pointers, column indices and values as vectors; one core,
// the block covering every row (no row-index compression).
template <typename F, typename I1, typename I2, typename I3, typename I4>
struct csr_matrix {
    typedef F float_type;
    typedef I1 row_idx_type;
    typedef I2 col_idx_type;
    vector::vector row, col, val, row_ind, col_ind;
    mem::sharing sharing_mode = mem::CORE;
    uint64_t nrows = 0, ncols = 0, nonzeros = 0;
    uint64_t block_nrows = 0, block_ncols = 0;
    uint64_t block_row_offset = 0, block_col_offset = 0;
    bool if_empty = false;
    bool if_indexed = false;
    const vector::vector &get_row_ind_vector() const { return row_ind; }
    // storage for nrows rows and `nonzeros` entries (the generators fill it)
    void alloc() {
        row.alloc_and_get_aligned_ptr<I1>(nrows + 1, 1);
        col.alloc_and_get_aligned_ptr<I2>(nonzeros, 1);
        val.alloc_and_get_aligned_ptr<F>(nonzeros, 1);
    }
    // row nrow's entries in the given order (rows filled in sequence)
    void upload_row(uint64_t nrow, const std::vector<uint64_t> &c, const std::vector<F> &v, uint32_t size) {
        I1 *rp = row.template get_aligned_ptr<I1>();
        I2 *cp = col.template get_aligned_ptr<I2>();
        F *vp = val.template get_aligned_ptr<F>();
        if (!nrow) rp[0] = 0;
        for (uint32_t i = 0; i < size; ++i) {
            cp[rp[nrow] + i] = (I2)c[i];
            vp[rp[nrow] + i] = v[i];
        }
        rp[nrow + 1] = rp[nrow] + size;
    }
};

template <typename F> struct dense_matrix {
    vector::vector val;
    mem::sharing sharing_mode = mem::CORE;
    uint64_t nrows = 0, ncols = 0;
    uint64_t block_nrows = 0, block_ncols = 0;
    uint64_t block_row_offset = 0, block_col_offset = 0;
    bool if_empty = false;
    dense_matrix() = default;
    explicit dense_matrix(mem::sharing m) : sharing_mode(m) {}
    // storage for nrows x ncols values, row-major
    void alloc() {
        val.alloc_and_get_aligned_ptr<F>(nrows * ncols, 1);
        if_empty = (nrows * ncols == 0);
    }
};

// The distributed matrix: only the members that the distributed inverse in
// operations/inverse.inl names (that routine itself is never instantiated
// here; its single-process core, the dense Gauss-Jordan inverse, is).
enum segmentation_type { SEGMENT_BY_BLOCKS, SEGMENT_BY_SLICES };
struct part_layer {
    std::vector<uint32_t> block_size = std::vector<uint32_t>(1, 0);
};
struct partitioning {
    part_layer node_layer, numa_layer;
};
struct matrix_block {
    int data = 0;  // the block's operator (a placeholder: never read here)
    bool reduced_prec = false;
    template <typename M> void assemble(M &, int) {}
    void get_inv_sqrt_diag() {}
    void get_inv_diag() {}
};
struct matrix_layer {
    matrix_block diag;
    std::vector<matrix_block> offd;
};
struct matrix_info_stub {
    void print(const std::string &, bool = false) const {}
    void print_header() const {}
    void print_footer() const {}
};

// One process's operator for the solver classes: a CSR block over caller
// arrays (the type-erased products of blas2.h reduce to one csr_Ax_y here),
// its spectrum bounds and D^{-1/2}.
struct matrix {
    std::map<segment::hierarchy, matrix_layer> data_layer;
    bool reduced_prec = false;
    segmentation_type segmentation = SEGMENT_BY_BLOCKS;
    partitioning *row_part = nullptr;
    float64_t min_eig = 0, max_eig = 0;
    matrix_info_stub info;
    int64_t n = 0, ncols = 0;
    const int *rp = nullptr, *ci = nullptr;
    const double *v = nullptr;
    std::vector<float> v32;   // FP32 values (reduced levels)
    vector::vector isd, invd;
    int nb = 1;               // hybrid Gauss-Seidel blocks (one per core)
    std::vector<int64_t> bp;  // their row offsets
    void set_part(partitioning *p) { row_part = p; }
    void add_data_layer(segment::hierarchy h) { data_layer[h]; }
    const vector::vector &inv_sqrt_diag() const { return isd; }
    const vector::vector &inv_diag() const { return invd; }
    template <typename F> void construct_core_layer() {}
};
// mg_layer (matrix.h:447-461): a level's operators and work vectors
struct mg_layer {
    matrix A, R, P;
    std::vector<vector::vector> buffer;
    matrix &get_A() { return A; }
    matrix &get_R() { return R; }
    matrix &get_P() { return P; }
};

}  // namespace matrix

// Declarations of the BLAS-1 templates whose definitions the included loop
// files provide (their signatures are those of src/blas/blas.h:47-130).
namespace blas {
template <typename T, const uint16_t NV> inline void copy(const vector::vector &x, vector::vector &y);
template <typename T, const uint16_t NV>
inline void bxor_global(const vector::vector &x, vector::vector &res);
template <typename T, const uint16_t NV>
inline void dot_global(const vector::vector &x, const vector::vector &y, vector::vector &res,
                       bool force = false);
template <typename T, const uint16_t NV>
inline void dot(const vector::vector &x, const vector::vector &y, vector::vector &res,
                bool force = false);
template <typename T, const uint16_t NV>
inline void vector_norm(const vector::vector &x, const uint16_t &norm_type, vector::vector &res,
                        bool force = false);
template <typename T, const uint16_t NV>
inline void set_const(vector::vector &x, const vector::vector &val, bool force = false);
template <typename T, const uint16_t NV> inline void set_rand(vector::vector &x, bool true_rand = false);
template <typename T, const uint16_t NV>
inline void ax_y(const vector::vector &a, const vector::vector &x, vector::vector &y);
template <typename T, const uint16_t NV>
inline void axpby(const vector::vector &a, const vector::vector &x, const vector::vector &b,
                  vector::vector &y);
template <typename T, const uint16_t NV> inline void scal(const vector::vector &x, vector::vector &y);
template <typename T, typename I, const uint16_t NV>
inline void gather(const vector::vector &x, const vector::indx_vector &indx, vector::vector &y,
                   bool force = true);
template <typename T, const uint16_t NV>
inline void forced_set_const(const vector::vector &x, const vector::vector &val);
template <typename T, const uint16_t NV>
inline void axpby_z(const vector::vector &a, const vector::vector &x, const vector::vector &b,
                    const vector::vector &y, vector::vector &z);
template <typename T, const uint16_t NV>
inline void axpbypcz(const vector::vector &a, const vector::vector &x, const vector::vector &b,
                     const vector::vector &y, const vector::vector &c, vector::vector &z);
template <typename T, const uint16_t NV>
inline void xdivy_z(const vector::vector &x, const vector::vector &y, vector::vector &z);
template <typename T, const uint16_t NV>
inline void upload(vector::vector &x, const T *ptr, uint64_t proc_size, uint64_t proc_offset);
template <typename T, const uint16_t NV> inline void pwr(vector::vector &x, const float64_t deg);
template <typename T> inline void set_const(vector::vector &x, const T a);
template <typename T, const uint16_t NV>
inline void set_const(vector::vector &x, const T val, bool force = false);
template <typename T, const uint16_t NV>
inline void set_const(vector::vector &x, const std::vector<T> &a, bool force = false);
template <typename T, const uint16_t NV> inline void forced_set_const(const vector::vector &x, const T val);
template <typename T, const uint16_t NV>
inline void axpby(const T a, const vector::vector &x, const T b, vector::vector &y);
}  // namespace blas

}  // namespace XAMG

// one of each per translation unit (internal linkage): the units of one
// library are compiled with different flags and share no symbol
static XAMG::perf_info perf;
static ID id;
