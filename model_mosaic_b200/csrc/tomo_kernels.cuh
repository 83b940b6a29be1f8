// Launchers shared between the translation units of the USFFT Radon pair.
#pragma once

#include <cuda_runtime.h>

namespace mmtomo {

// Length-2n transforms along v of the slice-interleaved spectrum, (n+1)*zs
// columns wide (tomo_col.cu), for 2n = 4096 and zs a multiple of 8.
// Forward (inv = false): src = Y, only the centre rows [n/2, 3n/2) are read,
// rows beyond radius n + 16 of the spectrum origin are not stored.  Inverse:
// src = F, rows beyond that radius are read as zeros, only the centre rows are
// stored.  The caller owns the scratch (col_fft_sizes: one L2-resident region
// per SM) and the twiddle table (filled by col_fft_twiddles on the host).
// Both return kNotCovered when (n, zs) is outside the kernel's range.
constexpr int kNotCovered = -100;
int col_fft_sizes(int n, int zs, int sms, size_t* scratch_elems, size_t* tw_elems);
void col_fft_twiddles(float2* tw);
int col_fft_pipe(int n, int zs, bool inv, const float2* src, float2* dst, float2* scratch, const float2* twl,
                 int sms, cudaStream_t st);

}  // namespace mmtomo
