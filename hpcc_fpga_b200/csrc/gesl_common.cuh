// Shared constants of the substitution kernels (k_gesl.cu, k_gesl_inv.cu).
#pragma once

#include "lp_common.cuh"

namespace lp {
namespace gesl {

constexpr int SB = 128;
constexpr int GT = 256;            // threads per CTA

}  // namespace gesl
}  // namespace lp
