// Times the reference's own GPU kernel on this machine's GPU.
//
// TEST INFRASTRUCTURE ONLY (a comparator, never part of the product): the cubins it loads
// are the reference's src/service/gpu/kernel.cu compiled unmodified by nvcc from the
// reference tree (oracle/Makefile target `ref_gpu`), one per field variant and batch, the
// way the reference's host compiles it at run time with NVRTC (src/service/gpu.rs:1355-1380:
// -DMEIKEY_BATCH, -DMEIKEY_FIELD, -DMEIKEY_UNPACKED).  This program drives them as the
// reference's host does:
//   - the comb table of width W in the reference's layout (src/service/gpu.rs:1416-1480: packed
//     8 words per coordinate, or 10 limbs for the unpacked R25 / K26 variants), built here by
//     the C oracle's restatement of the reference's builder;
//   - meikey_derive over one block of 32 threads, both seed sources, compared key by key with
//     the oracle before a variant is timed (the reference's Kernel::self_check,
//     src/service/gpu.rs:706-745);
//   - meikey_search with the reference's arguments and launch shape (src/service/gpu.rs:856-886):
//     block 128, grid = SMs x the occupancy of the kernel at 128 threads, keys_per_iter =
//     grid x 128 x batch, stop_on_hit = 0 (the reference's bench mode), iterations per
//     launch chosen so that a launch takes about 200 ms (TARGET_LAUNCH, gpu.rs:427), and
//     the rate timed with CUDA events over several such launches.
//
// Usage: ref_gpu <cubin-dir> <variants> <widths> <seconds-per-config>
//   variants: comma list of <limbs>_b<batch> with limbs 10, 10u, 8, 10k, 10ku, 5f
//   widths:   comma list of comb widths (2..20)
// Prints one JSON line per (variant, width, workload).
#include <cuda.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <thread>
#include <vector>

extern "C" {
void mko_init(void);
uint64_t mko_ref_table_words(uint32_t w);
void mko_ref_table_row(uint32_t w, uint32_t row, uint32_t* out);
void mko_derive(const uint8_t key[32], uint32_t src, uint64_t first, uint64_t n, uint8_t* out);
}

namespace {

#define CK(call)                                                                        \
    do {                                                                                \
        CUresult r_ = (call);                                                           \
        if (r_ != CUDA_SUCCESS) {                                                       \
            const char* s_ = nullptr;                                                   \
            cuGetErrorString(r_, &s_);                                                  \
            fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #call, s_ ? s_ : "?"); \
            exit(2);                                                                    \
        }                                                                               \
    } while (0)

struct Variant {
    std::string code;  // limbs code of the reference (Limbs::code, src/service/gpu.rs:86-95)
    uint32_t batch;
    bool unpacked() const { return code == "10u" || code == "10ku"; }
    bool k26() const { return code == "10k" || code == "10ku"; }
};

// comb table of width w: packed (24 words per entry) straight from the oracle, or converted to
// the 10-limb form of an unpacked variant (32 words per entry: 3 x 10 limbs and 2 words of
// padding), limb i of R25 at bit ceil(51 i / 2) with 26 / 25 bits, of K26 at bit 26 i with 26
std::vector<uint32_t> table_of(uint32_t w, int layout /*0 packed, 1 R25, 2 K26*/) {
    const uint64_t rows = (251 + w - 1) / w, cols = (1ull << (w - 1)) + 1;
    std::vector<uint32_t> packed(mko_ref_table_words(w));
    std::vector<std::thread> th;
    for (uint64_t r = 0; r < rows; r++)
        th.emplace_back([&, r] { mko_ref_table_row(w, (uint32_t)r, packed.data() + r * cols * 24); });
    for (auto& t : th) t.join();
    if (layout == 0) return packed;
    std::vector<uint32_t> out(rows * cols * 32, 0);
    for (uint64_t e = 0; e < rows * cols; e++)
        for (int f = 0; f < 3; f++) {
            const uint32_t* v = &packed[e * 24 + f * 8];
            auto bits = [&](unsigned start, unsigned len) -> uint32_t {
                unsigned q = start / 32, r = start % 32;
                uint64_t x = v[q];
                if (q + 1 < 8) x |= (uint64_t)v[q + 1] << 32;
                return (uint32_t)((x >> r) & ((1ull << len) - 1));
            };
            for (unsigned i = 0; i < 10; i++) {
                const unsigned start = layout == 1 ? (51 * i + 1) / 2 : 26 * i;
                const unsigned len = layout == 1 ? (i % 2 == 0 ? 26 : 25) : 26;
                out[e * 32 + f * 10 + i] = bits(start, len);
            }
        }
    return out;
}

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void key_words(const uint8_t key[32], uint32_t w[8]) {
    for (int i = 0; i < 8; i++)
        w[i] = (uint32_t)key[4 * i] | (uint32_t)key[4 * i + 1] << 8 | (uint32_t)key[4 * i + 2] << 16 |
               (uint32_t)key[4 * i + 3] << 24;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        fprintf(stderr, "usage: %s <cubin-dir> <variants> <widths> <seconds>\n", argv[0]);
        return 1;
    }
    const std::string dir = argv[1];
    std::vector<Variant> variants;
    for (char* t = strtok(argv[2], ","); t; t = strtok(nullptr, ",")) {
        std::string s(t);
        size_t b = s.find("_b");
        variants.push_back({s.substr(0, b), (uint32_t)atoi(s.c_str() + b + 2)});
    }
    std::vector<uint32_t> widths;
    for (char* t = strtok(argv[3], ","); t; t = strtok(nullptr, ",")) widths.push_back((uint32_t)atoi(t));
    const double seconds = atof(argv[4]);
    mko_init();
    CK(cuInit(0));
    CUdevice dev;
    CK(cuDeviceGet(&dev, 0));
    CUcontext ctx;
    CK(cuDevicePrimaryCtxRetain(&ctx, dev));
    CK(cuCtxSetCurrent(ctx));
    int sms = 0;
    CK(cuDeviceGetAttribute(&sms, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, dev));
    char name[128];
    CK(cuDeviceGetName(name, sizeof name, dev));
    CUstream st;
    CK(cuStreamCreate(&st, CU_STREAM_NON_BLOCKING));
    CUevent e0, e1;
    CK(cuEventCreate(&e0, CU_EVENT_DEFAULT));
    CK(cuEventCreate(&e1, CU_EVENT_DEFAULT));
    const uint32_t BLOCK = 128;  // src/service/gpu.rs:421

    // the workloads: the reference's published GPU mode (counter seeds, needle TARGET
    // case-insensitive, docs/benchmark.md) and the secure-path throughput configuration
    // (ChaCha20 seeds, case-sensitive 7-character contains)
    struct Work {
        const char* name;
        uint32_t counter;
        std::string needle;
        uint32_t fold;
        uint8_t key[32];
    };
    std::vector<Work> works = {{"counter/TARGET", 1, "target", 1, {}}, {"chacha20/8or5lx1", 0, "8or5lx1", 0, {}}};
    for (int i = 0; i < 32; i++) {
        works[0].key[i] = (uint8_t)(0x5a ^ (i * 29));
        works[1].key[i] = (uint8_t)(0xa5 ^ (i * 53));
    }

    for (uint32_t w : widths) {
        std::vector<CUdeviceptr> tables(3, 0);
        for (const Variant& v : variants) {
            const int layout = v.unpacked() ? (v.k26() ? 2 : 1) : 0;
            if (!tables[layout]) {
                std::vector<uint32_t> t = table_of(w, layout);
                CK(cuMemAlloc(&tables[layout], t.size() * 4));
                CK(cuMemcpyHtoD(tables[layout], t.data(), t.size() * 4));
            }
            const std::string path = dir + "/ref_" + v.code + "_b" + std::to_string(v.batch) + ".cubin";
            CUmodule mod;
            if (cuModuleLoad(&mod, path.c_str()) != CUDA_SUCCESS) {
                printf("{\"variant\": \"%s_b%u\", \"width\": %u, \"error\": \"cannot load %s\"}\n", v.code.c_str(),
                       v.batch, w, path.c_str());
                continue;
            }
            CUfunction search, derive;
            CK(cuModuleGetFunction(&search, mod, "meikey_search"));
            CK(cuModuleGetFunction(&derive, mod, "meikey_derive"));
            int occ = 0, regs = 0, local = 0;
            CK(cuOccupancyMaxActiveBlocksPerMultiprocessor(&occ, search, BLOCK, 0));
            CK(cuFuncGetAttribute(&regs, CU_FUNC_ATTRIBUTE_NUM_REGS, search));
            CK(cuFuncGetAttribute(&local, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, search));
            const uint32_t grid = (uint32_t)sms * (uint32_t)(occ > 0 ? occ : 1);
            const uint64_t kpi = (uint64_t)grid * BLOCK * v.batch;
            CUdeviceptr table = tables[layout];
            // self-check: 32 threads of meikey_derive from an odd index, both seed sources
            bool ok = true;
            {
                const uint32_t threads = 32;
                const uint64_t n = (uint64_t)threads * v.batch;
                CUdeviceptr d_key, d_out;
                CK(cuMemAlloc(&d_key, 32));
                CK(cuMemAlloc(&d_out, n * 32));
                for (uint32_t counter = 0; counter < 2 && ok; counter++) {
                    uint8_t key[32];
                    for (int i = 0; i < 32; i++) key[i] = (uint8_t)(i * 7 + counter * 91 + w);
                    uint32_t kw[8];
                    key_words(key, kw);
                    CK(cuMemcpyHtoD(d_key, kw, 32));
                    uint64_t first = 0x123456789ull * (w + 1) | 1;
                    void* args[] = {&table, &w, &d_key, &counter, &first, &d_out};
                    CK(cuLaunchKernel(derive, 1, 1, 1, threads, 1, 1, 0, st, args, nullptr));
                    CK(cuStreamSynchronize(st));
                    std::vector<uint8_t> got(n * 32), want(n * 32);
                    CK(cuMemcpyDtoH(got.data(), d_out, n * 32));
                    mko_derive(key, counter, first, n, want.data());
                    ok = got == want;
                }
                cuMemFree(d_key);
                cuMemFree(d_out);
            }
            for (const Work& wk : works) {
                if (!ok) break;
                CUdeviceptr d_key, d_needle, d_result, d_sink;
                uint32_t kw[8];
                key_words(wk.key, kw);
                CK(cuMemAlloc(&d_key, 32));
                CK(cuMemcpyHtoD(d_key, kw, 32));
                std::vector<uint8_t> nb(wk.needle.begin(), wk.needle.end());
                nb.resize(nb.size() + 64, 0);  // the reference pads the needle by 64 bytes
                CK(cuMemAlloc(&d_needle, nb.size()));
                CK(cuMemcpyHtoD(d_needle, nb.data(), nb.size()));
                CK(cuMemAlloc(&d_result, 16));
                CK(cuMemsetD8(d_result, 0, 16));
                CK(cuMemAlloc(&d_sink, (size_t)grid * BLOCK * 4));
                uint32_t counter = wk.counter, len = (uint32_t)wk.needle.size(), fold = wk.fold, mode = 0, stop = 0;
                uint64_t base = 0;
                uint32_t iters = 1;
                void* args[] = {&table, &w, &d_key, &counter, &d_needle, &len, &fold, &mode,
                                &base, &iters, &stop, &d_result, &d_sink};
                auto launch = [&](uint32_t it, uint64_t b) {
                    iters = it;
                    base = b;
                    CK(cuLaunchKernel(search, grid, 1, 1, BLOCK, 1, 1, 0, st, args, nullptr));
                };
                // warm-up and calibration to launches of about 200 ms
                launch(1, 0);
                CK(cuStreamSynchronize(st));
                double t = now_s();
                launch(1, kpi);
                CK(cuStreamSynchronize(st));
                const double once = now_s() - t;
                uint32_t it = (uint32_t)std::max(1.0, std::min(65536.0, 0.2 / std::max(once, 1e-6)));
                const int launches = std::max(1, (int)(seconds / 0.2 + 0.5));
                CK(cuEventRecord(e0, st));
                for (int l = 0; l < launches; l++) launch(it, kpi * (2 + (uint64_t)l * it));
                CK(cuEventRecord(e1, st));
                CK(cuEventSynchronize(e1));
                float ms = 0;
                CK(cuEventElapsedTime(&ms, e0, e1));
                const double keys = (double)kpi * it * launches;
                printf("{\"device\": \"%s\", \"variant\": \"%s_b%u\", \"limbs\": \"%s\", \"batch\": %u, \"width\": %u, "
                       "\"workload\": \"%s\", \"grid\": %u, \"block\": %u, \"blocks_per_sm\": %d, \"regs\": %d, "
                       "\"local_bytes\": %d, \"iters\": %u, \"launches\": %d, \"ms\": %.3f, \"keys_per_s\": %.6e, "
                       "\"self_check\": true}\n",
                       name, v.code.c_str(), v.batch, v.code.c_str(), v.batch, w, wk.name, grid, BLOCK, occ, regs, local,
                       it, launches, ms, keys / (ms * 1e-3));
                fflush(stdout);
                cuMemFree(d_key);
                cuMemFree(d_needle);
                cuMemFree(d_result);
                cuMemFree(d_sink);
            }
            if (!ok)
                printf("{\"variant\": \"%s_b%u\", \"width\": %u, \"self_check\": false}\n", v.code.c_str(), v.batch, w);
            cuModuleUnload(mod);
        }
        for (CUdeviceptr t : tables)
            if (t) cuMemFree(t);
    }
    cuDevicePrimaryCtxRelease(dev);
    return 0;
}
