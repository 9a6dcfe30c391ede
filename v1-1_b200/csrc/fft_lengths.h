// FFT lengths of the Coulomb passes: (P, P1, P2) with P = P1 * P2, two factors
// small enough for the register transforms; the plan picks the smallest P >= 2N-1.
#pragma once

#define SINCGPU_FFT_LENGTHS(X) \
  X(16, 4, 4) X(20, 5, 4) X(24, 6, 4) X(27, 9, 3) X(32, 8, 4) X(36, 6, 6) X(42, 7, 6) \
  X(48, 8, 6) X(54, 9, 6) X(64, 8, 8) X(72, 9, 8) X(81, 9, 9) X(90, 10, 9) X(100, 10, 10) \
  X(108, 12, 9) X(120, 12, 10) X(126, 14, 9) X(144, 12, 12) X(162, 18, 9) X(180, 15, 12) \
  X(192, 16, 12) X(216, 18, 12) X(240, 16, 15) X(256, 16, 16)

namespace sincgpu {

#define SINCGPU_LEN_ENTRY(P, A, B) P,
constexpr int kFftLens[] = {SINCGPU_FFT_LENGTHS(SINCGPU_LEN_ENTRY)};
#undef SINCGPU_LEN_ENTRY
constexpr int kNumFftLens = (int)(sizeof(kFftLens) / sizeof(kFftLens[0]));

// offset of length P's roots in the concatenated table of all lengths
constexpr int root_offset(int P) {
  int o = 0;
  for (int i = 0; i < kNumFftLens; ++i) {
    if (kFftLens[i] == P) return o;
    o += kFftLens[i];
  }
  return -1;
}
constexpr int root_total() {
  int o = 0;
  for (int i = 0; i < kNumFftLens; ++i) o += kFftLens[i];
  return o;
}

// Every translation unit that runs register transforms registers a function
// that uploads its own copy of the constant twiddle tables; contexts call all of
// them once per device before their first transform.
int register_const_roots(int (*upload)());
int upload_const_roots(int device);

}  // namespace sincgpu
