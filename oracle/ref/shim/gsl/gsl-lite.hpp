// Minimal stand-in for gsl-lite 0.42 used only to compile the reference's own
// proposal / cusparse2 sources into the test oracle (oracle/_ref).  The
// reference uses exactly one gsl symbol, gsl::narrow_cast, which is a plain
// static_cast.
#pragma once
namespace gsl {
template<class T, class U>
__host__ __device__ constexpr T narrow_cast(U&& u) noexcept {
    return static_cast<T>(static_cast<U&&>(u));
}
} // namespace gsl
