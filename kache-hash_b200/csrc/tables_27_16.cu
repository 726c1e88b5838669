// The engine's tables of 27-mers with 16-minimizers, one per value width.
#include "engine.cuh"

namespace kache_b200
{

kache_table* make_table_27_16(const uint32_t vb, const uint64_t n, const double lf, const bool pow2)
{
    switch(vb)
    {
    case 0: return new Engine<27, 16, void>(n, lf, pow2);
    case 1: return new Engine<27, 16, uint8_t>(n, lf, pow2);
    case 2: return new Engine<27, 16, uint16_t>(n, lf, pow2);
    case 4: return new Engine<27, 16, uint32_t>(n, lf, pow2);
    case 8: return new Engine<27, 16, uint64_t>(n, lf, pow2);
    default: return nullptr;
    }
}

}
