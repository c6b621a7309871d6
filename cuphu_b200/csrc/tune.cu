/*
 * tune.cu -- launch-shape autotuner state.
 *
 * cuphu_autotune (api.cu) times the candidate launch shapes of the cost
 * kernel and of the persistent solver on a caller's scene and stores the
 * fastest here, per device, kind and job-size class (floor(log2) of the
 * element count).  The launchers read the stored choice; a probing run
 * forces a candidate through tune_force.  CUPHU_TUNE=0 in the environment
 * makes the launchers ignore stored choices.
 */
#include <cstdlib>
#include <mutex>

#include "kernels.cuh"

namespace cuphu {
namespace {
/* kinds: 0 cost kernel variant, 1 mixed-precision solver shape, 2 FP64
 * solver shape (the shape indices of the two precisions differ) */
constexpr int kDevs = 64, kKinds = 3, kClasses = 48;
std::mutex g_tune_mu;
int g_tune[kDevs][kKinds][kClasses];
bool g_tune_init = false;
thread_local int g_force[kKinds] = {-1, -1, -1};
thread_local long long g_probe_items = 0;

void init_locked()
{
    if (g_tune_init) return;
    for (auto &d : g_tune)
        for (auto &k : d)
            for (int &c : k) c = -1;
    g_tune_init = true;
}
}  // namespace

int tune_class(long long n)
{
    int c = 0;
    while (n > 1 && c < kClasses - 1) {
        n >>= 1;
        ++c;
    }
    return c;
}

int tune_get(int dev, int kind, long long n)
{
    if (kind < 0 || kind >= kKinds) return -1;
    if (g_force[kind] >= 0) return g_force[kind];
    static const bool off = [] {
        const char *e = std::getenv("CUPHU_TUNE");
        return e && e[0] == '0';
    }();
    if (off || dev < 0 || dev >= kDevs) return -1;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    init_locked();
    return g_tune[dev][kind][tune_class(n)];
}

void tune_set(int dev, int kind, long long n, int v)
{
    if (dev < 0 || dev >= kDevs || kind < 0 || kind >= kKinds) return;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    init_locked();
    g_tune[dev][kind][tune_class(n)] = v;
}

void tune_force(int kind, int v)
{
    if (kind >= 0 && kind < kKinds) g_force[kind] = v;
}

void tune_note_items(long long n) { g_probe_items = n; }
long long tune_probe_items() { return g_probe_items; }

}  // namespace cuphu
