// wave_k7.cu -- schedule-4 wave kernel instances for padded disparity count 448;
// one translation unit per width keeps the build parallel.
#include "wave_inst.cuh"

LUMEN_WAVE_INSTANCE(7)
