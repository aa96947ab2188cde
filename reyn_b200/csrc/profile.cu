// Launch accounting behind REYN_KERNEL: per kernel name, the number of
// launches and (while enabled) the summed device time between a pair of CUDA
// events recorded around each launch on its stream.
#include "engine.cuh"

#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace reyn {
namespace {

struct Pending {
    int name;
    cudaEvent_t a, b;
};

struct Registry {
    std::mutex mu;
    std::atomic<bool> timing { false };
    std::vector<std::string> names;
    std::map<std::string, int> index;
    std::vector<uint64_t> launches;
    std::vector<double> ms;
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;

    int id(const char* n)
    {
        auto it = index.find(n);
        if (it != index.end())
            return it->second;
        const int k = (int)names.size();
        names.emplace_back(n);
        index.emplace(n, k);
        launches.push_back(0);
        ms.push_back(0.0);
        return k;
    }
    cudaEvent_t event()
    {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        REYN_CUDA(cudaEventCreate(&e));
        return e;
    }
    // folds finished event pairs into the totals (synchronising on them)
    void drain()
    {
        for (auto& p : pending) {
            REYN_CUDA(cudaEventSynchronize(p.b));
            float t = 0.f;
            REYN_CUDA(cudaEventElapsedTime(&t, p.a, p.b));
            ms[p.name] += t;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
};

Registry& reg()
{
    static Registry* r = new Registry(); // outlives every static destructor
    return *r;
}

thread_local int t_open = -1; // index into pending of the open scope
thread_local std::vector<const char*>* t_sink = nullptr; // capture: names only

} // namespace

void profile_record(std::vector<const char*>* sink) { t_sink = sink; }

ProfScope::ProfScope(const char* name, cudaStream_t s)
    : s_(s)
{
    if (t_sink) { // captured into a graph: the replay counts it
        t_sink->push_back(name);
        return;
    }
    Registry& r = reg();
    std::lock_guard<std::mutex> lock(r.mu);
    const int k = r.id(name);
    r.launches[k] += 1;
    if (!r.timing.load(std::memory_order_relaxed))
        return;
    Pending p { k, r.event(), r.event() };
    REYN_CUDA(cudaEventRecord(p.a, s));
    r.pending.push_back(p);
    slot_ = (int)r.pending.size() - 1;
}

ProfScope::~ProfScope()
{
    if (slot_ < 0)
        return;
    Registry& r = reg();
    std::lock_guard<std::mutex> lock(r.mu);
    if (slot_ < (int)r.pending.size())
        cudaEventRecord(r.pending[slot_].b, s_);
}

// counts `times` launches of each named kernel (graph replays)
void profile_count(const std::vector<const char*>& names, uint64_t times)
{
    if (!times)
        return;
    Registry& r = reg();
    std::lock_guard<std::mutex> lock(r.mu);
    for (const char* n : names)
        r.launches[r.id(n)] += times;
}

} // namespace reyn

extern "C" {

int reyn_profile_enable(int on)
{
    return reyn::guard([&] { reyn::reg().timing.store(on != 0); });
}

int reyn_profile_reset(void)
{
    return reyn::guard([&] {
        auto& r = reyn::reg();
        std::lock_guard<std::mutex> lock(r.mu);
        r.drain();
        std::fill(r.launches.begin(), r.launches.end(), 0);
        std::fill(r.ms.begin(), r.ms.end(), 0.0);
    });
}

int reyn_profile_read(reyn_profile_entry* out, uint32_t cap, uint32_t* count)
{
    return reyn::guard([&] {
        reyn::require(count != nullptr, "null count");
        auto& r = reyn::reg();
        std::lock_guard<std::mutex> lock(r.mu);
        r.drain();
        uint32_t k = 0;
        for (size_t i = 0; i < r.names.size(); ++i) {
            if (!r.launches[i])
                continue;
            if (out && k < cap) {
                std::memset(out[k].name, 0, sizeof(out[k].name));
                std::strncpy(out[k].name, r.names[i].c_str(), sizeof(out[k].name) - 1);
                out[k].launches = r.launches[i];
                out[k].total_ms = r.ms[i];
            }
            ++k;
        }
        *count = k;
    });
}

} // extern "C"
