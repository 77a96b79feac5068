// Status reporting of the specula_b200 C ABI.
#include "sb_common.cuh"

namespace sb {

static thread_local char g_last_error[512] = "";

int fail(int status, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

void clear_error() { g_last_error[0] = '\0'; }

}  // namespace sb

extern "C" int sb_version(void) { return 100; }

extern "C" const char *sb_last_error(void) { return sb::g_last_error; }

// ---- TMA tensor maps and device properties (declared in sb_tma.cuh) ----
#include "sb_tma.cuh"

namespace sb {

namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
}  // namespace

int tensor_map_2d_f32(CUtensorMap *map, const float *base, int rows, int cols, int ld, int box_rows, int box_cols) {
    static EncodeTiledFn enc = nullptr;
    if (!enc) {
        cudaDriverEntryPointQueryResult qr;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) != cudaSuccess ||
            qr != cudaDriverEntryPointSuccess || !fn)
            return fail(SB_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
        enc = reinterpret_cast<EncodeTiledFn>(fn);
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || ((size_t)ld * 4) % 16 || ((size_t)box_cols * 4) % 16)
        return fail(SB_EINVAL, "tensor map: base, row stride and box width must be 16-byte multiples");
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(SB_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SB_OK;
}

int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        cache[dev] = n;
    }
    return cache[dev];
}

}  // namespace sb

// ---------------------------------------------------------------------------
// Tile-shape tuning registry: (kernel family, shape key) -> variant.
// ---------------------------------------------------------------------------
#include <map>
#include <mutex>
#include <utility>

namespace {
std::mutex g_tune_mutex;
std::map<std::pair<int, unsigned long long>, int> g_tune;
const char *const kDmBatchedVariants[] = {
    "16 realisations per pass, 1 mode-row group", "16 realisations per pass, 2 mode-row groups",
    "8 realisations per pass, 1 mode-row group",  "8 realisations per pass, 2 mode-row groups",
    "4 realisations per pass, 1 mode-row group",  "4 realisations per pass, 2 mode-row groups",
    "8 realisations per pass, 4 columns per thread, 1024-column tiles",
    "8 realisations per pass, 4 columns per thread, 512-column tiles",
    "8 realisations per pass, 4 columns per thread, 256-column tiles",
    "16 realisations per pass, 4 columns per thread, 1024-column tiles",
    "16 realisations per pass, 4 columns per thread, 512-column tiles",
    "16 realisations per pass, 4 columns per thread, 256-column tiles"};
const char *const kShFp32Variants[] = {"8 sub-apertures per CTA, field tile by TMA",
                                       "4 sub-apertures per CTA, field tile by TMA",
                                       "2 sub-apertures per CTA, field tile by TMA", "8 sub-apertures per CTA",
                                       "4 sub-apertures per CTA", "2 sub-apertures per CTA"};
const char *const kModalrecVariants[] = {"2 reconstructor rows per CTA", "1 reconstructor row per CTA",
                                         "4 reconstructor rows per CTA"};
}  // namespace

namespace sb {
int tune_lookup(int family, unsigned long long key) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune.find({family, key});
    return it == g_tune.end() ? 0 : it->second;
}
}  // namespace sb

extern "C" int sb_tune_variants(int family) {
    switch (family) {
        case SB_TUNE_DM_BATCHED: return (int)(sizeof(kDmBatchedVariants) / sizeof(kDmBatchedVariants[0]));
        case SB_TUNE_SH_FP32: return (int)(sizeof(kShFp32Variants) / sizeof(kShFp32Variants[0]));
        case SB_TUNE_MODALREC_BATCHED: return (int)(sizeof(kModalrecVariants) / sizeof(kModalrecVariants[0]));
        default: return 0;
    }
}

extern "C" const char *sb_tune_variant_name(int family, int variant) {
    if (variant < 0 || variant >= sb_tune_variants(family)) return "";
    switch (family) {
        case SB_TUNE_DM_BATCHED: return kDmBatchedVariants[variant];
        case SB_TUNE_SH_FP32: return kShFp32Variants[variant];
        default: return kModalrecVariants[variant];
    }
}

extern "C" unsigned long long sb_tune_key(int a, int b, int c) {
    return ((unsigned long long)(unsigned)a << 40) ^ ((unsigned long long)(unsigned)b << 12) ^
           (unsigned long long)(unsigned)c;
}

extern "C" int sb_tune_set(int family, unsigned long long key, int variant) {
    sb::clear_error();
    const int n = sb_tune_variants(family);
    if (n == 0) return sb::fail(SB_EINVAL, "sb_tune_set: unknown kernel family %d", family);
    if (variant >= n) return sb::fail(SB_EINVAL, "sb_tune_set: family %d has %d variants", family, n);
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    if (variant < 0)
        g_tune.erase({family, key});
    else
        g_tune[{family, key}] = variant;
    return SB_OK;
}

extern "C" int sb_tune_get(int family, unsigned long long key) {
    if (sb_tune_variants(family) == 0) return -1;
    return sb::tune_lookup(family, key);
}
