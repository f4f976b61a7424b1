// Where a pointer argument of the C ABI lives, decided from its CUDA pointer
// attributes.  Kept free of CUDA headers so that the rule can be checked on a
// machine without a GPU (the CPU tests compile it with g++).
#pragma once

namespace tosp {

enum PtrKind {
    PTR_HOST = 0,           // pageable or pinned host memory: staged through the handle's buffers
    PTR_DEVICE = 1,         // memory the handle's kernels may read and write directly
    PTR_OTHER_DEVICE = -1,  // device memory of another GPU: refused (no peer access is set up)
};

// Memory-type codes of cudaPointerAttributes::type (cudaMemoryType).
constexpr int MEMTYPE_UNREGISTERED = 0, MEMTYPE_HOST = 1, MEMTYPE_DEVICE = 2, MEMTYPE_MANAGED = 3;

// attrs_ok: cudaPointerGetAttributes succeeded; mem_type / mem_device: its
// type and device fields; handle_device: the device the handle was created on.
inline int classify_ptr(bool attrs_ok, int mem_type, int mem_device, int handle_device) {
    if (!attrs_ok) return PTR_HOST;
    if (mem_type == MEMTYPE_DEVICE) return mem_device == handle_device ? PTR_DEVICE : PTR_OTHER_DEVICE;
    if (mem_type == MEMTYPE_MANAGED) return PTR_DEVICE;   // migrates on access from any device
    return PTR_HOST;
}

}  // namespace tosp
