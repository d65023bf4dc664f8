// Host construction of the float32 sincos exception table (see acb_sincos_table_build_host in
// include/acoular_b200.h).
//
// The reference's map kernel (acoular/fastFuncs.py:260-261) rounds the phase k*r to float32 and
// evaluates cos/sin in float32 through the C library (cosf/sinf).  The device kernels compute the
// correctly rounded float32 cos/sin of the same float32 argument via FP64 evaluation.  The two
// agree on ~99.8 % of arguments; this table lists the others, obtained by calling the host
// library's cosf/sinf and the host's FP64 cos/sin on every float32 in [0, max_arg).  Nothing
// about the library's implementation is used -- only its outputs.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "../../include/acoular_b200.h"

namespace {

struct Exc {
    uint32_t key;
    int8_t dcos, dsin;
};

inline int32_t fbits(float f)
{
    int32_t i;
    memcpy(&i, &f, 4);
    return i;
}

void scan(uint32_t lo, uint32_t hi, std::vector<Exc> *out, int *overflow)
{
    for (uint32_t b = lo; b < hi; ++b) {
        float x;
        memcpy(&x, &b, 4);
        const float cg = cosf(x), sg = sinf(x);
        const float cr = (float)cos((double)x), sr = (float)sin((double)x);
        const int32_t dc = fbits(cg) - fbits(cr), ds = fbits(sg) - fbits(sr);
        if (dc == 0 && ds == 0) continue;
        if (dc < -127 || dc > 127 || ds < -127 || ds > 127 || ((fbits(cg) ^ fbits(cr)) < 0 && dc) ||
            ((fbits(sg) ^ fbits(sr)) < 0 && ds)) {
            ++*overflow;
            continue;
        }
        out->push_back(Exc{b, (int8_t)dc, (int8_t)ds});
    }
}

}  // namespace

extern "C" int64_t acb_sincos_table_build_host(uint64_t *table_host, int64_t slots, float max_arg, int num_threads)
{
    if (!table_host || slots < (1 << 16) || (slots & (slots - 1)) || !(max_arg > 0.f)) return -ACB_ERR_ARG;
    if (num_threads <= 0) num_threads = (int)std::max(1u, std::thread::hardware_concurrency());
    uint32_t hi_bits;
    memcpy(&hi_bits, &max_arg, 4);
    std::vector<std::vector<Exc>> parts(num_threads);
    std::vector<int> overflow(num_threads, 0);
    std::vector<std::thread> th;
    const uint64_t chunk = (hi_bits + (uint64_t)num_threads - 1) / num_threads;
    for (int t = 0; t < num_threads; ++t) {
        const uint32_t lo = (uint32_t)std::min<uint64_t>(hi_bits, t * chunk);
        const uint32_t hi = (uint32_t)std::min<uint64_t>(hi_bits, (t + 1) * chunk);
        th.emplace_back(scan, lo, hi, &parts[t], &overflow[t]);
    }
    for (auto &x : th) x.join();
    int64_t n = 0;
    for (int t = 0; t < num_threads; ++t) {
        if (overflow[t]) return -ACB_ERR_UNSUPPORTED;
        n += (int64_t)parts[t].size();
    }
    if (n * 2 > slots) return -ACB_ERR_SHAPE;  // keep the load factor below 1/2
    const uint64_t mask = (uint64_t)slots - 1;
    std::fill(table_host, table_host + slots, ~0ull);
    for (auto &p : parts)
        for (const Exc &e : p) {
            uint64_t slot = ((uint64_t)e.key * 0x9E3779B97F4A7C15ull) >> 20;
            int probes = 0;
            while (table_host[slot & mask] != ~0ull) {
                ++slot;
                // the device lookup gives up after 64 probes; a longer chain would hide entries
                if (++probes >= 63) return -ACB_ERR_SHAPE;
            }
            table_host[slot & mask] =
                ((uint64_t)e.key << 32) | ((uint64_t)(uint8_t)e.dcos << 8) | (uint64_t)(uint8_t)e.dsin;
        }
    return n;
}
