// Unit-kernel shapes with 16x16 blocks.
#include "inst_unit.cuh"

namespace dft2h {

Variant unit_variant_b16(int T, int NW, int MINB) {
    DFT2_UNIT_SHAPE(16, 1, 16, 1)
    DFT2_UNIT_SHAPE(16, 3, 10, 2)
    DFT2_UNIT_SHAPE(16, 5, 12, 1)
    DFT2_UNIT_SHAPE(16, 7, 8, 1)
    DFT2_UNIT_SHAPE(16, 1, 8, 2)
    DFT2_UNIT_SHAPE(16, 3, 8, 2)
    DFT2_UNIT_SHAPE(16, 3, 16, 1)
    DFT2_UNIT_SHAPE(16, 3, 4, 4)
    return Variant{};
}

}  // namespace dft2h
