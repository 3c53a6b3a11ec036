// Per-kernel timing with CUDA events on the launching stream, for the roofline report.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "baking_b200.h"
#include "bk_common.h"
#include "bk_profile.h"

namespace {

struct Record {
    int name;
    cudaEvent_t start, end;
};

std::mutex g_mutex;
bool g_enabled = false;
std::string g_only;  // when not empty, only the kernel of this name is recorded
std::vector<std::string> g_names;
std::vector<Record> g_records;
std::vector<cudaEvent_t> g_free;

cudaEvent_t take_event() {
    if (!g_free.empty()) {
        cudaEvent_t e = g_free.back();
        g_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

}  // namespace

int bk::profile_begin(const char* name, cudaStream_t stream) {
    if (!g_enabled) return -1;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_only.empty() && g_only != name) return -1;
    int id = -1;
    for (size_t k = 0; k < g_names.size(); ++k)
        if (g_names[k] == name) id = (int)k;
    if (id < 0) {
        g_names.emplace_back(name);
        id = (int)g_names.size() - 1;
    }
    Record r{id, take_event(), take_event()};
    if (!r.start || !r.end) return -1;
    cudaEventRecord(r.start, stream);
    g_records.push_back(r);
    return (int)g_records.size() - 1;
}

void bk::profile_end(int record, cudaStream_t stream) {
    if (record < 0) return;
    std::lock_guard<std::mutex> lock(g_mutex);
    cudaEventRecord(g_records[record].end, stream);
}

extern "C" {

int bk_profile_start(void) {
    std::lock_guard<std::mutex> lock(g_mutex);
    for (auto& r : g_records) {
        g_free.push_back(r.start);
        g_free.push_back(r.end);
    }
    g_records.clear();
    g_names.clear();
    g_enabled = true;
    return BK_OK;
}

int bk_profile_select(const char* name) {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_only = name ? name : "";
    return BK_OK;
}

int bk_profile_stop(void) {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_enabled = false;
    return BK_OK;
}

int bk_profile_report(int32_t max_kernels, char* names, int32_t name_capacity, double* total_ms, int32_t* counts,
                      int32_t* kernel_count) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!names || !total_ms || !counts || !kernel_count || max_kernels <= 0 || name_capacity <= 0)
        return bk::fail(BK_ERR_ARGUMENT, "bk_profile_report: bad arguments");
    int k_count = (int)g_names.size() < max_kernels ? (int)g_names.size() : max_kernels;
    for (int k = 0; k < k_count; ++k) {
        total_ms[k] = 0.0;
        counts[k] = 0;
        std::strncpy(names + (size_t)k * name_capacity, g_names[k].c_str(), name_capacity - 1);
        names[(size_t)k * name_capacity + name_capacity - 1] = '\0';
    }
    for (const Record& r : g_records) {
        if (r.name >= k_count) continue;
        if (cudaEventSynchronize(r.end) != cudaSuccess) return bk::fail(BK_ERR_LAUNCH, "bk_profile_report: event failed");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.start, r.end);
        total_ms[r.name] += ms;
        counts[r.name] += 1;
    }
    *kernel_count = k_count;
    return BK_OK;
}

}  // extern "C"
