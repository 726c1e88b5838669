// The engine's tables of 32-mers with 20-minimizers, one per value width.
#include "engine.cuh"

namespace kache_b200
{

kache_table* make_table_32_20(const uint32_t vb, const uint64_t n, const double lf, const bool pow2)
{
    switch(vb)
    {
    case 0: return new Engine<32, 20, void>(n, lf, pow2);
    case 1: return new Engine<32, 20, uint8_t>(n, lf, pow2);
    case 2: return new Engine<32, 20, uint16_t>(n, lf, pow2);
    case 4: return new Engine<32, 20, uint32_t>(n, lf, pow2);
    case 8: return new Engine<32, 20, uint64_t>(n, lf, pow2);
    default: return nullptr;
    }
}

}
