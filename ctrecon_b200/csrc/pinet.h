// pinet.h -- constants of the learned PI-line initialiser (pinet.cu, pinet_infer.cu).
#pragma once

#include <cstdint>

namespace ctr {

constexpr int kPinetH = 64;         // hidden width
constexpr int kPinetParams = 12866; // 3->64->64->64->64->2 weights and biases
constexpr int kPinetParamsPad = 12868;
constexpr double kPinetRInv = 4.0;       // feature 0 = r * 4 (r normalised by ScanR)
constexpr double kPinetOutScale = 4.0;   // outputs are 4x the endpoint offsets (radians)

// layer l = 0..4: fan-in, fan-out, and the offsets of W_l[out][in] (row-major) and b_l[out]
// in the parameter vector
__host__ __device__ constexpr int pinet_in(int l) { return l == 0 ? 3 : 64; }
__host__ __device__ constexpr int pinet_out(int l) { return l == 4 ? 2 : 64; }
__host__ __device__ constexpr int pinet_offW(int l) {
    return l == 0 ? 0 : l == 1 ? 256 : l == 2 ? 4416 : l == 3 ? 8576 : 12736;
}
__host__ __device__ constexpr int pinet_offB(int l) {
    return l == 0 ? 192 : l == 1 ? 4352 : l == 2 ? 8512 : l == 3 ? 12672 : 12864;
}

// inference buffer: W_1..W_3 of the hidden 64x64 layers as BF16 [out][in] (3 x 8 KB), then FP32
// values: W_0 (BF16-rounded, 192), b_0..b_3 (4 x 64), W_4 (BF16-rounded, 128), b_4 (2)
constexpr int kNetBf16Bytes = 3 * 64 * 64 * 2;
constexpr int kNetF32 = 192 + 4 * 64 + 128 + 2;
constexpr int kNetBytes = kNetBf16Bytes + kNetF32 * 4;
constexpr int kNetF32_W0 = 0, kNetF32_B0 = 192, kNetF32_W4 = 448, kNetF32_B4 = 576;

}  // namespace ctr
