// search_flat_ch3.cu -- flat-search kernels for rows of up to 96 neighbours (3 chunk(s) of 32).
#include "search_flat_kernels.cuh"

namespace pgb {
void* flat_kernel_ch3(FlatSchedule sched, bool is_signed, uint32_t filter_words) {
    return flat_kernel_ch<3>(sched, is_signed, filter_words);
}
cudaError_t flat_section_totals_ch3(unsigned long long* acc, bool reset) {
    return flat_section_totals(acc, reset);
}
}  // namespace pgb
