// Unit-kernel shapes with 32x32 blocks.
#include "inst_unit.cuh"

namespace dft2h {

Variant unit_variant_b32(int T, int NW, int MINB) {
    DFT2_UNIT_SHAPE(32, 1, 16, 1)
    DFT2_UNIT_SHAPE(32, 1, 8, 1)
    DFT2_UNIT_SHAPE(32, 3, 6, 2)
    DFT2_UNIT_SHAPE(32, 3, 8, 1)
    DFT2_UNIT_SHAPE(32, 3, 4, 2)
    DFT2_UNIT_SHAPE(32, 5, 5, 1)
    DFT2_UNIT_SHAPE(32, 5, 6, 1)
    DFT2_UNIT_SHAPE(32, 5, 7, 1)
    DFT2_UNIT_SHAPE(32, 7, 5, 1)
    return Variant{};
}

}  // namespace dft2h
