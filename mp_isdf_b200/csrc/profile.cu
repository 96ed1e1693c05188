// Per-kernel-family CUDA-event timing, off by default.  When enabled, every
// instrumented launch site records an event pair on its own stream; reading
// the profile synchronises those events and sums elapsed times per family.
#include "../../include/isdf_b200.h"
#include "isdf_internal.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>

namespace isdf {
namespace {

struct Record {
    const char* name;
    cudaEvent_t a, b;
};

std::atomic<bool> g_enabled{false};
std::mutex g_mu;
std::vector<Record> g_records;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    ISDF_CUDA(cudaEventCreate(&e));
    return e;
}

}  // namespace

bool profiling_enabled() { return g_enabled.load(std::memory_order_relaxed); }

namespace {
std::atomic<int64_t> g_launches{0};
}  // namespace

void count_launches(int64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

ProfileScope::ProfileScope(const char* name, cudaStream_t s) : name_(name), s_(s) {
    if (!profiling_enabled()) return;
    std::lock_guard<std::mutex> lk(g_mu);
    a_ = take_event();
    b_ = take_event();
    ISDF_CUDA(cudaEventRecord(a_, s_));
}

ProfileScope::~ProfileScope() {
    if (!a_) return;
    if (cudaEventRecord(b_, s_) != cudaSuccess) return;
    std::lock_guard<std::mutex> lk(g_mu);
    g_records.push_back({name_, a_, b_});
}

}  // namespace isdf

extern "C" {

int64_t isdf_launch_count(void) { return isdf::g_launches.load(std::memory_order_relaxed); }

int isdf_profile_enable(int32_t on) {
    isdf::g_enabled.store(on != 0);
    return ISDF_OK;
}

int isdf_profile_read(int32_t max, char* names, double* total_ms, int64_t* launches, int32_t* count) {
    std::lock_guard<std::mutex> lk(isdf::g_mu);
    std::map<std::string, std::pair<double, int64_t>> acc;
    int status = ISDF_OK;
    for (auto& r : isdf::g_records) {
        float ms = 0;
        if (cudaEventSynchronize(r.b) != cudaSuccess || cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess)
            status = ISDF_ERR_CUDA;
        auto& e = acc[r.name];
        e.first += ms;
        e.second += 1;
        isdf::g_pool.push_back(r.a);
        isdf::g_pool.push_back(r.b);
    }
    isdf::g_records.clear();
    std::vector<std::pair<std::string, std::pair<double, int64_t>>> v(acc.begin(), acc.end());
    std::sort(v.begin(), v.end(), [](auto& x, auto& y) { return x.second.first > y.second.first; });
    const int n = std::min<int>(max, static_cast<int>(v.size()));
    for (int i = 0; i < n; ++i) {
        if (names) {
            std::memset(names + 48 * i, 0, 48);
            std::strncpy(names + 48 * i, v[i].first.c_str(), 47);
        }
        if (total_ms) total_ms[i] = v[i].second.first;
        if (launches) launches[i] = v[i].second.second;
    }
    if (count) *count = n;
    return status;
}

}  // extern "C"
