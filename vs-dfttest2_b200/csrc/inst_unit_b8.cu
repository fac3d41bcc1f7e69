// Unit-kernel shapes with 8x8 blocks.
#include "inst_unit.cuh"

namespace dft2h {

Variant unit_variant_b8(int T, int NW, int MINB) {
    DFT2_UNIT_SHAPE(8, 1, 16, 1)
    DFT2_UNIT_SHAPE(8, 3, 16, 1)
    DFT2_UNIT_SHAPE(8, 5, 16, 1)
    DFT2_UNIT_SHAPE(8, 7, 16, 1)
    DFT2_UNIT_SHAPE(8, 1, 8, 2)
    DFT2_UNIT_SHAPE(8, 3, 8, 2)
    return Variant{};
}

}  // namespace dft2h
