// Launch counter and per-pass event timing (see instrument.cuh).
#include <mutex>
#include <vector>
#include "../../include/ifdda_gpu.h"
#include "instrument.cuh"

namespace ifdda {

std::atomic<unsigned long long>& launch_counter() {
    static std::atomic<unsigned long long> c{0};
    return c;
}

namespace {
struct Timing {
    std::mutex mu;
    int pass = PASS_NONE;
    int prec_bytes = 0;  // 0: any precision, else sizeof(complex) of the timed kernels
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pairs;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
};
Timing& timing() {
    static Timing t;
    return t;
}
}  // namespace

cudaEvent_t timing_before(int pass, int precision_bytes, cudaStream_t st) {
    Timing& t = timing();
    if (t.pass == PASS_NONE || pass != t.pass) return nullptr;
    if (t.prec_bytes && t.prec_bytes != precision_bytes) return nullptr;
    std::lock_guard<std::mutex> lk(t.mu);
    cudaEvent_t a = t.get();
    cudaEventRecord(a, st);
    return a;
}

bool timing_active() { return timing().pass != PASS_NONE; }

void timing_after(cudaEvent_t start, cudaStream_t st) {
    if (!start) return;
    Timing& t = timing();
    std::lock_guard<std::mutex> lk(t.mu);
    cudaEvent_t b = t.get();
    cudaEventRecord(b, st);
    t.pairs.emplace_back(start, b);
}

}  // namespace ifdda

using namespace ifdda;

extern "C" {

unsigned long long ifdda_launch_count(void) { return launch_counter().load(); }

int ifdda_timing_enable(int pass, int precision) {
    Timing& t = timing();
    std::lock_guard<std::mutex> lk(t.mu);
    t.pass = pass;
    t.prec_bytes = precision == IFDDA_FP64 ? 16 : precision == IFDDA_FP32 ? 8 : 0;
    for (auto& p : t.pairs) {
        t.pool.push_back(p.first);
        t.pool.push_back(p.second);
    }
    t.pairs.clear();
    return 0;
}

int ifdda_timing_read(int* launches, double* total_ms) {
    Timing& t = timing();
    std::lock_guard<std::mutex> lk(t.mu);
    double tot = 0;
    int n = 0;
    for (auto& p : t.pairs) {
        if (cudaEventSynchronize(p.second) != cudaSuccess) return 1;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, p.first, p.second) != cudaSuccess) return 1;
        tot += ms;
        n++;
        t.pool.push_back(p.first);
        t.pool.push_back(p.second);
    }
    t.pairs.clear();
    if (launches) *launches = n;
    if (total_ms) *total_ms = tot;
    return 0;
}

}  // extern "C"
