// Build-recipe support only: oneDAL runtime services that the table and
// descriptor sources reference but that a client of the k-means path never
// needs (TBB-backed threading loops, CPU feature detection). In a full oneDAL
// build these come from oneDAL itself.
#include "services/env_detect.h"

#include <cstddef>
#include <cstdint>

namespace daal { namespace services { namespace interface1 {
int Environment::getStatus() { return 0; }
Environment *Environment::getInstance() { return nullptr; }
int Environment::getCpuId(int) { return 0; }
}}}  // namespace daal::services::interface1

int __daal_serv_cpu_detect(int) { return 0; }
bool daal_check_is_intel_cpu() { return false; }
int daal_enabled_cpu_detect() { return 0; }
uint64_t daal_serv_cpu_feature_detect() { return 0; }

namespace daal { typedef void (*functype)(int i, const void *a); }
extern "C" void _daal_threader_for(int n, int, const void *a, daal::functype f) {
    for (int i = 0; i < n; ++i) f(i, a);
}

typedef void (*loop_i64)(std::int64_t, const void *);
typedef void (*loop_blocked)(std::size_t, std::size_t, const void *);
extern "C" {
void _onedal_threader_for_int64(std::int64_t n, const void *a, loop_i64 f) {
    for (std::int64_t i = 0; i < n; ++i) f(i, a);
}
void _onedal_threader_for_blocked_size(std::size_t n, std::size_t b, const void *a, loop_blocked f) {
    for (std::size_t s = 0; s < n; s += b) f(s, s + b < n ? s + b : n, a);
}
}
