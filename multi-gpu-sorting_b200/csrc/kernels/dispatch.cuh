// Maps the C ABI's mgs_dtype to the KeyTraits instantiation that implements it.
#pragma once

#include "device_common.cuh"

namespace mgs {

using TraitsU32 = KeyTraits<uint32_t, kUnsignedKey>;
using TraitsI32 = KeyTraits<uint32_t, kSignedKey>;
using TraitsF32 = KeyTraits<uint32_t, kFloatKey>;
using TraitsU64 = KeyTraits<unsigned long long, kUnsignedKey>;
using TraitsI64 = KeyTraits<unsigned long long, kSignedKey>;
using TraitsF64 = KeyTraits<unsigned long long, kFloatKey>;

// Calls fn(Traits{}) for the dtype; returns false for an unknown dtype.
template <typename Fn>
inline bool dispatch_dtype(int dtype, Fn&& fn) {
  switch (dtype) {
    case 0: fn(TraitsU32{}); return true;
    case 1: fn(TraitsI32{}); return true;
    case 2: fn(TraitsF32{}); return true;
    case 3: fn(TraitsU64{}); return true;
    case 4: fn(TraitsI64{}); return true;
    case 5: fn(TraitsF64{}); return true;
    default: return false;
  }
}

}  // namespace mgs
