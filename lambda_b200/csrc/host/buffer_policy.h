// Which caller-owned buffers an entry point that takes device pointers accepts.
//
// Plain integers stand for the CUDA runtime's cudaMemoryType (0 unregistered,
// 1 host, 2 device, 3 managed), so the rule compiles and is tested without the
// CUDA headers or a GPU.
#pragma once

namespace lambda_host {

enum MemoryKind { kMemUnregistered = 0, kMemHost = 1, kMemDevice = 2, kMemManaged = 3 };

// A buffer is usable by kernels on `device` when it is device memory of that same
// GPU, or managed memory (which migrates to the GPU that touches it). Device memory
// of another GPU is refused: without peer access a kernel that touched it would
// fault instead of the call returning an error.
inline bool buffer_usable_on(int kind, int owner_device, int device) {
    if (kind == kMemManaged) return true;
    return kind == kMemDevice && owner_device == device;
}

}  // namespace lambda_host
