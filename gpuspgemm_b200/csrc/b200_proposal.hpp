// Header-only C++ drop-in for the reference's entry point
//
//     template<std::floating_point T>
//     utils::DeviceCSR<T> proposal::proposal(const utils::DeviceCSR<T>& A,
//                                            const utils::DeviceCSR<T>& B);
//     (geektrove/GPUSpGEMM src/libproposal/include/proposal/proposal.cuh:85-124)
//
// b200::proposal(A, B) accepts any CSR type laid out like utils::CSR<T, Device>
// (public members nnz, m, n, rpt, col, val; default constructible; frees its
// arrays with cudaFree), including the reference's own utils::DeviceCSR<T>, and
// returns the same type owning library-allocated arrays (cudaMallocAsync, so
// the type's cudaFree releases them).  Errors throw std::runtime_error, as the
// reference's utils::handle_cuda_error does (errors.cuh:11-22).  In the
// reference's apps the swap is one line (src/apps/proposal.cu:25, 32):
//     return b200::proposal(d_a, d_b).template to<utils::Location::Host>();
#pragma once

#include <stdexcept>
#include <string>
#include <type_traits>

#include "spgemm.h"

namespace b200 {

// One handle per host thread (the C ABI's threading rule).
inline spgemm_handle_t thread_handle() {
    struct Holder {
        spgemm_handle_t h = nullptr;
        ~Holder() {
            if (h != nullptr) spgemm_destroy(h);
        }
    };
    thread_local Holder holder;
    if (holder.h == nullptr) {
        const spgemm_status st = spgemm_create(&holder.h, -1);
        if (st != SPGEMM_OK)
            throw std::runtime_error(std::string("spgemm_create: ") +
                                     spgemm_last_error_string());
    }
    return holder.h;
}

template<typename CSR>
CSR proposal(const CSR& A, const CSR& B, void* stream = nullptr) {
    using T = std::remove_cv_t<std::remove_pointer_t<decltype(A.val)>>;
    static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>,
                  "values must be float or double");
    const spgemm_csr_view va{A.m, A.n, A.nnz, A.rpt, A.col, A.val};
    const spgemm_csr_view vb{B.m, B.n, B.nnz, B.rpt, B.col, B.val};
    spgemm_csr_out out{};
    spgemm_status st;
    if constexpr (std::is_same_v<T, double>) {
        st = spgemm_csr_f64(thread_handle(), &va, &vb, &out, stream);
    } else {
        st = spgemm_csr_f32(thread_handle(), &va, &vb, &out, stream);
    }
    if (st != SPGEMM_OK)
        throw std::runtime_error(std::string(spgemm_status_string(st)) + ": " +
                                 spgemm_last_error_string());
    CSR C;
    C.nnz = out.nnz;
    C.m = out.m;
    C.n = out.n;
    C.rpt = out.rpt;
    C.col = out.col;
    C.val = static_cast<T*>(out.val);
    return C;
}

// Total intermediate products (reference utils::get_nip, nip.cuh:52-78).
template<typename CSR>
long long get_nip(const CSR& A, const CSR& B, void* stream = nullptr) {
    const spgemm_csr_view va{A.m, A.n, A.nnz, A.rpt, A.col, A.val};
    const spgemm_csr_view vb{B.m, B.n, B.nnz, B.rpt, B.col, B.val};
    int64_t nip = 0;
    const spgemm_status st = spgemm_get_nip(thread_handle(), &va, &vb, &nip, stream);
    if (st != SPGEMM_OK)
        throw std::runtime_error(std::string(spgemm_status_string(st)) + ": " +
                                 spgemm_last_error_string());
    return nip;
}

}  // namespace b200
