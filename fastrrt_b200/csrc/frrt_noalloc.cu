// frrt_noalloc.cu -- the kinematic candidate check without device allocation.
//
// fastrrt_candidates_kinematic_noalloc() runs the same kernels as a
// fastrrt_candidates_create() context followed by
// fastrrt_candidates_kinematic_device(), but it never calls cudaMalloc or
// cudaFree: callers such as a real-time control loop whose device memory is
// reserved up front, a process under a memory-pool policy that forbids new
// device allocations, or code that must not reach the driver's allocator
// while other work is in flight can still call it.  Its working memory (the
// instance record and the three bit-packed frame masks) lives in one
// file-scope __device__ array, sized for frames up to 1024 x 1024 cells and
// kept by every GPU that loads the library until the process exits.  The
// array's device address is looked up once per device and kept: a process
// that calls cudaDeviceReset must not call this entry point afterwards on
// that device (the reloaded module may place the array elsewhere).
#include <cmath>
#include <cstring>
#include <mutex>

#include "fastrrt_b200.h"
#include "frrt_engine.h"
#include "frrt_kernels.cuh"

using namespace frrt;

namespace {

constexpr int kNoAllocMaxW = 1024;
constexpr int kNoAllocMaxH = 1024;
constexpr int kNoAllocMaxDevices = 64;
constexpr int kNoAllocMaxClasses = 256;  // class ids are uint8
// words of one bit-packed mask of the largest frame (a multiple of 4)
constexpr size_t kMaskWordsMax = (size_t)((kNoAllocMaxW + 31) / 32) * kNoAllocMaxH;
constexpr size_t kInstOffset = 0;
constexpr size_t kStateOffset = 1024;
constexpr size_t kSlotOffset = 1536;     // one int: the slot list {0}
constexpr size_t kBadOffset = 1540;      // one int: class id outside the cost table
constexpr size_t kBadCellOffset = 1544;  // one int: candidate start cell outside the frame
constexpr size_t kMaskOffset = 2048;     // blocked, clear, dilation scratch
constexpr size_t kScratchBytes = kMaskOffset + 3 * 4 * kMaskWordsMax;
static_assert(sizeof(Inst) <= kStateOffset - kInstOffset, "instance record exceeds its space");
static_assert(sizeof(State) <= kSlotOffset - kStateOffset, "state record exceeds its space");
static_assert(kMaskWordsMax % 4 == 0, "masks must stay 16-byte aligned");

struct DeviceScratch {
    unsigned char *base;  // device address of g_noalloc_scratch on this device
    int sms;
};
DeviceScratch g_dev[kNoAllocMaxDevices];
std::mutex g_mutex;

}  // namespace

// Host code must not use this name as a device address: in host code it is a
// host-side stand-in.  The address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

// Once per device, with that device current: the array's device address and
// the multiprocessor count.  No allocation.
bool scratch_for_current_device(DeviceScratch &out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("candidates_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return false;
    }
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error("candidates_noalloc: device index out of range");
        return false;
    }
    DeviceScratch &d = g_dev[dev];
    if (!d.base) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("candidates_noalloc: cudaGetSymbolAddress: ") +
                      cudaGetErrorString(e));
            return false;
        }
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess || sms <= 0) {
            set_error(std::string("candidates_noalloc: device query: ") + cudaGetErrorString(e));
            return false;
        }
        d.sms = sms;
        d.base = static_cast<unsigned char *>(p);
    }
    out = d;
    return true;
}

}  // namespace

extern "C" int fastrrt_candidates_kinematic_noalloc(
    int width, int height, const uint8_t *class_ids, const float *class_costs, int n_classes,
    const float *heading_grid, const float *cost_grid, int min_dist_x, int min_dist_z,
    int lowerBound_x, int lowerBound_z, int upperBound_x, int upperBound_z,
    double max_steering_rad, double lr_m, int n, const int32_t *sx, const int32_t *sz,
    const float *steer, const float *length, float velocity_m_s, float *out4, uint64_t *probes,
    void *stream)
{
    if (width <= 0 || height <= 0 || width > kNoAllocMaxW || height > kNoAllocMaxH) {
        set_error("candidates_noalloc: frame size must be 1..1024 x 1..1024 cells");
        return -1;
    }
    if (n_classes <= 0 || n_classes > kNoAllocMaxClasses || !class_ids || !class_costs || !heading_grid ||
        !cost_grid || min_dist_x < 0 || min_dist_z < 0 || n < 0 ||
        (n > 0 && (!sx || !sz || !steer || !length || !out4))) {
        set_error("candidates_noalloc: bad arguments");
        return -1;
    }
    if (n == 0)
        return 0;
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceScratch d;
    if (!scratch_for_current_device(d))
        return -1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char *base = d.base;
    Inst *d_inst = reinterpret_cast<Inst *>(base + kInstOffset);
    State *d_state = reinterpret_cast<State *>(base + kStateOffset);
    int *d_slots = reinterpret_cast<int *>(base + kSlotOffset);
    int *d_bad = reinterpret_cast<int *>(base + kBadOffset);
    int *d_bad_cell = reinterpret_cast<int *>(base + kBadCellOffset);
    uint32_t *masks = reinterpret_cast<uint32_t *>(base + kMaskOffset);

    // the instance record a candidates context would hold for this frame
    Inst I;
    memset(&I, 0, sizeof(Inst));
    I.W = width;
    I.H = height;
    I.mask_rw = (width + 31) / 32;
    I.mask_words = (I.mask_rw * height + 3) / 4 * 4;
    I.og_x = (float)(width / 2);
    I.og_z = (float)(height / 2);
    I.cls = class_ids;
    I.class_costs = class_costs;
    I.n_classes = n_classes;
    I.blocked = masks;
    I.clear = masks + kMaskWordsMax;
    I.rowdil = masks + 2 * kMaskWordsMax;
    I.trav = nullptr;
    I.heading = const_cast<float *>(heading_grid);  // read only
    I.cost = const_cast<float *>(cost_grid);        // read only
    I.intrinsic = nullptr;
    I.max_steer = max_steering_rad;
    I.lr = lr_m;
    I.lbx = lowerBound_x;
    I.lbz = lowerBound_z;
    I.ubx = upperBound_x;
    I.ubz = upperBound_z;
    I.mdx = (int)((float)min_dist_x / 2);
    I.mdz = (int)((float)min_dist_z / 2);
    I.rc = (int)std::floor(std::sqrt((double)I.mdx * I.mdx + (double)I.mdz * I.mdz)) + 2;

    // every call shares the array: the record, the state, the slot list and
    // the error flag are written afresh before any kernel reads them
    cudaError_t e = cudaMemcpyAsync(d_inst, &I, sizeof(Inst), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(base + kStateOffset, 0, kMaskOffset - kStateOffset, st);
    if (e != cudaSuccess) {
        set_error(std::string("candidates_noalloc: ") + cudaGetErrorString(e));
        return -1;
    }
    launch_frame_masks(d_inst, d_state, d_slots, 1, I.mask_words, n_classes, d_bad, st);
    Launch L{};
    L.sms = d.sms;
    L.sweep_blocks = d.sms * 8;
    L.work_blocks = d.sms * 2;
    L.smem_words = 0;  // masks are read from the array (through L2), not staged
    launch_candidates(d_inst, 0, n, sx, sz, steer, length, velocity_m_s,
                      reinterpret_cast<float4 *>(out4), reinterpret_cast<unsigned long long *>(probes),
                      L, st, d_bad_cell);
    int bad[2] = {0, 0};  // class id flag, cell flag (adjacent ints)
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(bad, d_bad, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(std::string("candidates_noalloc: ") + cudaGetErrorString(e));
        return -1;
    }
    if (bad[0]) {
        set_error("candidates_noalloc: frame class id outside the class-cost table");
        return -1;
    }
    if (bad[1]) {
        set_error("candidates_noalloc: candidate start cell outside the frame");
        return -1;
    }
    return 0;
}
