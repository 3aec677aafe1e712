#pragma once
// Pinned host words for the engines' per-iteration read-backs: one pinned
// block per process, handed out in 64-byte slots.  A pinned allocation
// costs milliseconds, so graph::build makes it (before Run is timed); a
// read-back into pinned memory is a plain asynchronous copy, where one into
// ordinary memory goes through a staging buffer every iteration.

#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

namespace graph_one::detail {

class PinnedSlots {
public:
    static constexpr int kSlots = 64;
    static constexpr int kWords = 16;  // 64 bytes per slot

    static PinnedSlots& get() {
        static PinnedSlots p;  // process lifetime: never freed
        return p;
    }
    // A free slot, or null when none is left (or pinned memory failed).
    uint32_t* take() {
        std::lock_guard<std::mutex> lk(mu_);
        if (!base_) return nullptr;
        for (int i = 0; i < kSlots; ++i)
            if (!used_[i]) {
                used_[i] = true;
                return base_ + i * kWords;
            }
        return nullptr;
    }
    void give(uint32_t* s) {
        std::lock_guard<std::mutex> lk(mu_);
        if (base_ && s >= base_ && s < base_ + kSlots * kWords) used_[(s - base_) / kWords] = false;
    }

private:
    PinnedSlots() {
        void* p = nullptr;
        if (cudaHostAlloc(&p, kSlots * kWords * 4, cudaHostAllocDefault) == cudaSuccess)
            base_ = static_cast<uint32_t*>(p);
        else
            cudaGetLastError();
    }
    std::mutex mu_;
    uint32_t* base_ = nullptr;
    bool used_[kSlots] = {};
};

}  // namespace graph_one::detail
