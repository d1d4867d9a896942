// Internal declarations shared by the host-side sources of libspektri_b200.
#pragma once
#include <cstdint>

namespace sk {

int fail(int code, const char* fmt, ...);
void clear_error();

bool format_valid(int c);
bool format_complex(int c);
int format_bits(int c);
int format_bytes(int c);
float format_scaling(int c);

bool freq_to_bins(double fs, double fc, long long N, double fs_out, double fc_out, long long* bins, long long* first);
void bins_to_freq(double fs, double fc, long long N, long long bins, long long first, double* fs_out, double* fc_out);
bool freq_to_bins_exact(double fs, double fc, long long N, double fs_out, double fc_out, long long* bins, long long* first);
void raised_cosine(uint32_t n, float* out_c64);
void tukey(uint32_t n, uint32_t tw, float* out_c64);

}  // namespace sk
