// search_flat_ch2.cu -- flat-search kernels for rows of up to 64 neighbours (2 chunk(s) of 32).
#include "search_flat_kernels.cuh"

namespace pgb {
void* flat_kernel_ch2(FlatSchedule sched, bool is_signed, uint32_t filter_words) {
    return flat_kernel_ch<2>(sched, is_signed, filter_words);
}
cudaError_t flat_section_totals_ch2(unsigned long long* acc, bool reset) {
    return flat_section_totals(acc, reset);
}
}  // namespace pgb
