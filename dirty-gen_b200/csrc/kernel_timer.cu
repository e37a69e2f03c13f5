// Per-launch device timing of this library's kernels (silt_set_kernel_timing).
//
// While timing is on, launch_ex records one CUDA event on the launch's stream
// before the launch and one after it; silt_get_kernel_times waits for the
// device, books each pair's elapsed time to its kernel and returns the totals
// by kernel. The events sit between launches, so a timed run loses the
// launch overlap of programmatic dependent launches: time a separate pass,
// not the run whose throughput is reported.
#include <cuda_runtime.h>
#include <cxxabi.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "launch_count.cuh"
#include "../../include/silt_sheet.h"

namespace silt {
namespace {

struct Pair {
    const void* kernel;
    cudaEvent_t a, b;
};

struct Timer {
    std::mutex m;
    std::vector<cudaEvent_t> pool;
    std::vector<Pair> pending;
    std::map<const void*, std::pair<long long, double>> totals;  // launches, ms
    cudaEvent_t take() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        return e;
    }
};

Timer g_timer;
std::atomic<bool> g_on{false};
thread_local cudaEvent_t t_open = nullptr;  // the event recorded before this thread's current launch

std::string kernel_name(const void* k) {
    const char* raw = nullptr;
    if (cudaFuncGetName(&raw, k) != cudaSuccess || !raw) {
        cudaGetLastError();
        return "unknown";
    }
    int st = 0;
    char* dem = abi::__cxa_demangle(raw, nullptr, nullptr, &st);
    std::string out = (st == 0 && dem) ? dem : raw;
    std::free(dem);
    // Keep the qualified name, drop the argument list (and anonymous
    // namespaces, whose parentheses would end the name early).
    const std::string anon = "(anonymous namespace)::";
    for (size_t at = out.find(anon); at != std::string::npos; at = out.find(anon)) out.erase(at, anon.size());
    const size_t paren = out.find('(');
    if (paren != std::string::npos) out.resize(paren);
    return out;
}

}  // namespace

bool kernel_timing_on() { return g_on.load(std::memory_order_relaxed); }

void kernel_timing_begin(cudaStream_t st) {
    std::lock_guard<std::mutex> lk(g_timer.m);
    t_open = g_timer.take();
    if (t_open && cudaEventRecord(t_open, st) != cudaSuccess) {
        g_timer.pool.push_back(t_open);
        t_open = nullptr;
    }
}

void kernel_timing_end(cudaStream_t st, const void* kernel) {
    std::lock_guard<std::mutex> lk(g_timer.m);
    if (!t_open) return;
    cudaEvent_t b = g_timer.take();
    if (b && cudaEventRecord(b, st) == cudaSuccess) {
        g_timer.pending.push_back(Pair{kernel, t_open, b});
    } else {
        g_timer.pool.push_back(t_open);
        if (b) g_timer.pool.push_back(b);
    }
    t_open = nullptr;
}

}  // namespace silt

extern "C" {

int silt_set_kernel_timing(int32_t on) {
    std::lock_guard<std::mutex> lk(silt::g_timer.m);
    if (on) {
        // A fresh run: earlier totals and unread pairs are dropped.
        for (const silt::Pair& p : silt::g_timer.pending) {
            silt::g_timer.pool.push_back(p.a);
            silt::g_timer.pool.push_back(p.b);
        }
        silt::g_timer.pending.clear();
        silt::g_timer.totals.clear();
    }
    silt::g_on.store(on != 0);
    return SILT_OK;
}

int silt_get_kernel_times(silt_kernel_time* out, int32_t cap, int32_t* n_out) {
    if (!n_out || cap < 0 || (cap > 0 && !out)) return SILT_EINVAL;
    if (cudaDeviceSynchronize() != cudaSuccess) return SILT_ECUDA;
    std::lock_guard<std::mutex> lk(silt::g_timer.m);
    for (const silt::Pair& p : silt::g_timer.pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            auto& t = silt::g_timer.totals[p.kernel];
            t.first += 1;
            t.second += ms;
        } else {
            cudaGetLastError();
        }
        silt::g_timer.pool.push_back(p.a);
        silt::g_timer.pool.push_back(p.b);
    }
    silt::g_timer.pending.clear();
    // Largest total first.
    std::vector<std::pair<const void*, std::pair<long long, double>>> rows(silt::g_timer.totals.begin(),
                                                                            silt::g_timer.totals.end());
    std::sort(rows.begin(), rows.end(), [](const auto& x, const auto& y) { return x.second.second > y.second.second; });
    int k = 0;
    for (const auto& r : rows) {
        if (k < cap) {
            silt_kernel_time& o = out[k];
            memset(&o, 0, sizeof o);
            const std::string name = silt::kernel_name(r.first);
            strncpy(o.name, name.c_str(), sizeof o.name - 1);
            o.launches = r.second.first;
            o.ms = r.second.second;
        }
        ++k;
    }
    *n_out = k;
    return SILT_OK;
}

}  // extern "C"
