// Factory of unit-kernel shapes, included by the per-block-size units
// inst_unit_b8.cu, inst_unit_b16.cu and inst_unit_b32.cu (each instantiates
// the kernels of one block size, so the three compile in parallel).
#pragma once

#include "dfttest_host.h"

namespace dft2h {

template <int B, int T, int NW, int MINB>
Variant make_unit_variant() {
    Variant v;
    v.main = dft2::dfttest_unit_kernel<B, T, NW, dft2::kFilterWiener, MINB>;
    v.generic = dft2::dfttest_unit_kernel<B, T, NW, dft2::kFilterGeneric, MINB>;
    v.fixup = dft2::dfttest_fixup_kernel<B>;
    v.nw = NW;
    v.bpw = 32 / B;
    v.minb = MINB;
    v.smem = [](int pitch) { return dft2::Layout<B, T, NW>::smem_bytes(pitch); };
    return v;
}

}  // namespace dft2h

// one `if` per compiled shape (T, warps per CTA, CTAs per SM)
#define DFT2_UNIT_SHAPE(B_, T_, NW_, MINB_) \
    if (T == T_ && NW == NW_ && MINB == MINB_) return make_unit_variant<B_, T_, NW_, MINB_>();
