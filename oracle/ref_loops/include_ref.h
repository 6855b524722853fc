// The reference's loop files, included unchanged from its source tree
// (the build recipe puts <reference>/src on the include path), after the
// stand-in types of shim.h.
#pragma once
#include "shim.h"

#include "blas/detail/blas.inl"
#include "blas/detail/blas_ext.inl"
#include "blas/detail/blas_wrapper.inl"
#include "blas/detail/specific/blas_merged_jacobi.inl"
#include "blas2/detail/csr_matvec.inl"
#include "blas2/detail/csr_gs.inl"
#include "blas2/detail/dense_matvec.inl"
#include "primitives/matrix/operations/inverse.inl"
#include "primitives/vector/operations/convert.inl"

namespace refloops {

using XAMG::vector::vector;

// Calls f.template operator()<NV>() for the runtime width nv; -1 if nv is
// not one of the instantiated widths.
template <class Fn> int dispatch_nv(int nv, Fn &&f) {
    switch (nv) {
    case 1: f.template run<1>(); return 0;
    case 2: f.template run<2>(); return 0;
    case 4: f.template run<4>(); return 0;
    case 8: f.template run<8>(); return 0;
    case 16: f.template run<16>(); return 0;
    case 32: f.template run<32>(); return 0;
    }
    return -1;
}

// Views of caller arrays as the reference's vector objects.
template <class T> vector block(const T *p, int64_t n, int nv) {
    vector v;
    v.view<T>(const_cast<T *>(p), (uint64_t)n, (uint16_t)nv);
    return v;
}

// per-column scalars: a vector of one row and nv columns
template <class T> vector scalars(const T *p, int nv) { return block<T>(p, 1, nv); }

}  // namespace refloops
