// common.cuh -- field layout, launch helpers and error plumbing shared by the kernels and the host
// orchestration of the B200 Kohn-Sham solver.
//
// Field layout in HBM (the "pitched cube"): a real-space field on the cubic n^3 grid is stored
// x-fastest with a row pitch P = n rounded up to a multiple of 4 floats (16 B):
//     element (i, j, k) at  (k*n + j)*P + i,     field stride F = n*n*P floats.
// There are no ghost cells: the Dirichlet zero outside the box comes from the TMA loads' out-of-
// bounds fill (the tensor map's extent is n on every axis), so a field costs n*n*P floats instead
// of the reference's (n+8)^3 (crates/qm-gpu/src/grid.rs:3-27). The pad columns i in [n, P) hold 0:
// kernels that generate a field write 0 there, arithmetic kernels map 0 to 0, and the reductions
// therefore sum the pads harmlessly. Blocks of fields (LOBPCG's X, W, P, ...) are contiguous with
// stride F, which makes one 4-D tensor map (n, n, n, count) cover a whole block.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace ks {

struct Layout {
    int n = 0;       // points per axis
    int P = 0;       // row pitch (floats), multiple of 4
    long long F = 0; // floats per field
    double h = 0;    // spacing (Bohr)
    double origin = 0; // coordinate of index 0 on every axis: -(n-1)h/2 (crates/qm/src/grid.rs:11-14)
    static Layout make(int n, double h) {
        Layout L;
        L.n = n;
        L.P = (n + 3) & ~3;
        L.F = (long long)n * n * L.P;
        L.h = h;
        L.origin = -((double)(n - 1) * h / 2.0);
        return L;
    }
    long long interior() const { return (long long)n * n * n; }
};

// A CUDA error inside the library becomes this exception; the C ABI turns it into KS_DEVICE.
struct DeviceError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// Broken numerics (NaN Gram, non-SPD CG, lost rank) become this; the C ABI maps it to KS_NUMERICAL.
struct NumericalError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void check_cuda(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        char buf[512];
        snprintf(buf, sizeof buf, "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
        throw DeviceError(buf);
    }
}
#define KS_CUDA(call) ::ks::check_cuda((call), #call, __FILE__, __LINE__)
// Every kernel launch of the library goes through this check, which also counts it
// (ks_launch_count: the number of this library's kernels launched by the process).
void count_launch();
// A CUDA graph replay adds its kernel nodes; while the calling thread captures a graph, its launches are not counted.
void count_launches(long long n);
void set_capturing(bool on);
#define KS_LAUNCH_CHECK() (::ks::count_launch(), ::ks::check_cuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__))

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Number of SMs of the current device (148 on B200), cached per device.
int sm_count();
// The device int that kernels with bounded waits set to nonzero when a wait gives up, as the calling host thread
// sees it at launch time: the flag an ErrorFlagScope installed on this thread (a solver's own for the duration of
// its calls, a kernel hook's own), else the device's shared flag, which the device-pointer entry points use and
// ks_device_status reads. A solver's flag is reset at the start of each solve and read with each readback, so a
// timeout is reported by the call whose kernels raised it and by no other solver.
int* device_error_flag();
class ErrorFlagScope {
public:
    explicit ErrorFlagScope(int* flag);
    ~ErrorFlagScope();
    ErrorFlagScope(const ErrorFlagScope&) = delete;
    ErrorFlagScope& operator=(const ErrorFlagScope&) = delete;

private:
    int* prev_;
};
// Synchronises s, reads the calling thread's current flag and clears it; throws DeviceError when a wait gave up.
void check_device_flag(cudaStream_t s);
// Zeroes fresh device memory and waits for it (cudaMemset on the legacy stream).
void zero_device(void* p, size_t bytes);

// An NVTX range over a scope: one phase of the solve (a solve, an SCF step, an eigensolve, a Poisson solve, the
// forces) as a profiler shows it, and what ncu --nvtx filters on. The ranges are per host thread, so the down channel's
// eigensolve on its own thread nests correctly; with no tool attached a range costs a function call.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Runs set() once per device for one call site (`done` holds a bit per device index): a kernel's
// function attributes (its dynamic shared-memory limit, the carveout) belong to the context of the
// device they were set on, so a solver on a second device of the same process sets them again.
// Two threads may both run set() the first time; setting an attribute twice is harmless.
template <class Set>
void once_per_device(std::atomic<unsigned long long>& done, Set&& set) {
    int dev = 0;
    KS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw DeviceError("device index out of range");
    const unsigned long long bit = 1ull << dev;
    if (done.load(std::memory_order_acquire) & bit) return;
    set();
    done.fetch_or(bit, std::memory_order_acq_rel);
}

}  // namespace ks
