// ouroboros_b200.cuh -- C++/CUDA drop-in for the reference's Ouroboros types.
//
// A program written against GPUPeople/Ouroboros
//
//     #include "device/Ouroboros_impl.cuh"
//     #include "device/MemoryInitialization.cuh"
//     #include "InstanceDefinitions.cuh"
//     MultiOuroPQ mm;  mm.initialize(8ull << 30);
//     kernel<<<g, b>>>(mm.getDeviceMemoryManager(), ...);   // mm->malloc(size), mm->free(ptr)
//
// switches to this build by including this header instead, linking
// libouroboros_b200.so (heap creation) and naming the types from namespace
// ouro.  The device side -- malloc/free inlined into the caller's kernel -- is
// the header-only ouro::Ouroboros<V>; include/ouroboros_b200.h is the C ABI.
#pragma once

#include <cstddef>
#include <stdexcept>

#include "../ouroboros_b200/csrc/ouro/ouroboros.cuh"
#include "ouroboros_b200.h"

namespace ouro {

// Host owner of one heap (Ouroboros<...> of include/device/Ouroboros.cuh:247-297).
// Move-only: the heap is freed once, by the owner.
template <int V>
class HostOuroboros {
 public:
  using DeviceType = Ouroboros<V>;

  HostOuroboros() = default;
  HostOuroboros(const HostOuroboros&) = delete;
  HostOuroboros& operator=(const HostOuroboros&) = delete;
  HostOuroboros(HostOuroboros&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
  HostOuroboros& operator=(HostOuroboros&& o) noexcept {
    if (this != &o) {
      release();
      h_ = o.h_;
      o.h_ = nullptr;
    }
    return *this;
  }
  ~HostOuroboros() { release(); }

  // MemoryInitialization.cuh:123-219; idempotent like the reference.  The two
  // extra reservations of the reference's signature are accepted and unused.
  void initialize(size_t instantiation_size, size_t /*additionalSizeBeginning*/ = 0,
                  size_t /*additionalSizeEnd*/ = 0) {
    if (h_) return;
    int rc = ouro_create(V, instantiation_size, &h_);
    if (rc != OURO_OK) throw std::runtime_error(ouro_status_string(rc));
  }

  // Ouroboros.cuh:297: the object device code calls malloc/free on.
  DeviceType* getDeviceMemoryManager() const { return static_cast<DeviceType*>(ouro_device_handle(h_)); }

  ouro_heap* handle() const { return h_; }

 private:
  void release() {
    if (h_) ouro_destroy(h_);
    h_ = nullptr;
  }
  ouro_heap* h_ = nullptr;
};

// include/InstanceDefinitions.cuh:16-34
using MultiOuroPQ = HostOuroboros<0>;
using MultiOuroCQ = HostOuroboros<1>;
using MultiOuroVAPQ = HostOuroboros<2>;
using MultiOuroVACQ = HostOuroboros<3>;
using MultiOuroVLPQ = HostOuroboros<4>;
using MultiOuroVLCQ = HostOuroboros<5>;

}  // namespace ouro
