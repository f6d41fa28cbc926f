// aprb_sample_image_noalloc: particle sampling for callers that must not
// allocate device memory while they run (real-time acquisition loops, plugin
// hosts with a fixed device-memory budget).  The down-sampling pyramid lives
// in a file-scope device array, reserved on a device when this module is
// first used there (at library load only with eager module loading); no
// cudaMalloc / cudaFree is called on this path.
#include <mutex>

#include "kernels.cuh"

namespace aprb {

// Pyramid scratch: 32 Mi uint16 values (64 MiB) per device that loads the library.
constexpr uint64_t kNoAllocScratchElems = uint64_t(32) << 20;
static __device__ __align__(256) uint16_t g_noalloc_scratch[kNoAllocScratchElems];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint16_t *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array for the current device, looked up with
// that device current.  A call outside stream capture looks it up again (a
// device reset reloads the module at another address); a call under capture
// uses the address of the last call on the device.
uint16_t *scratch_for_current_device(bool refresh) {
    int dev = 0;
    APRB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device ordinal out of range for the no-allocation scratch table");
        throw Error{APRB_ERR_INVALID_ARGUMENT};
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev] || refresh) {
        void *p = nullptr;
        APRB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_ptr[dev] = (uint16_t *)p;
    }
    return g_scratch_ptr[dev];
}

}  // namespace
}  // namespace aprb

using namespace aprb;

extern "C" aprb_status aprb_sample_image_noalloc(const uint64_t *xz_end_dev, const uint16_t *y_vec_dev, int y_num,
                                                 int x_num, int z_num, const uint16_t *img_dev, uint16_t *parts_dev,
                                                 void *stream) {
    try {
        if (!xz_end_dev || !y_vec_dev || !img_dev || !parts_dev || y_num < 1 || x_num < 1 || z_num < 1 ||
            y_num > 65535 || x_num > 65535 || z_num > 65535) {
            set_error("aprb_sample_image_noalloc: null pointer or invalid dimensions");
            return APRB_ERR_INVALID_ARGUMENT;
        }
        Geom g;
        apr_geometry(y_num, x_num, z_num, g);
        const uint64_t need = sample_scratch_elems(g);
        if (need > kNoAllocScratchElems) {
            set_error("aprb_sample_image_noalloc: the volume's sampling pyramid needs " + std::to_string(need) +
                      " uint16 values, more than the fixed scratch of " + std::to_string(kNoAllocScratchElems));
            return APRB_ERR_INVALID_ARGUMENT;
        }
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        APRB_CUDA(cudaStreamIsCapturing((cudaStream_t)stream, &cs));
        uint16_t *scratch = scratch_for_current_device(cs == cudaStreamCaptureStatusNone);
        launch_sample_scratch(g, xz_end_dev, y_vec_dev, img_dev, parts_dev, scratch, (cudaStream_t)stream);
        return APRB_OK;
    } catch (const Error &e) {
        return e.status;
    } catch (...) {
        set_error("aprb_sample_image_noalloc: unexpected exception");
        return APRB_ERR_CUDA;
    }
}
