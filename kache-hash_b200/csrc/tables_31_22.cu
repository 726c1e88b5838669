// The engine's tables of 31-mers with 22-minimizers, one per value width.
#include "engine.cuh"

namespace kache_b200
{

kache_table* make_table_31_22(const uint32_t vb, const uint64_t n, const double lf, const bool pow2)
{
    switch(vb)
    {
    case 0: return new Engine<31, 22, void>(n, lf, pow2);
    case 1: return new Engine<31, 22, uint8_t>(n, lf, pow2);
    case 2: return new Engine<31, 22, uint16_t>(n, lf, pow2);
    case 4: return new Engine<31, 22, uint32_t>(n, lf, pow2);
    case 8: return new Engine<31, 22, uint64_t>(n, lf, pow2);
    default: return nullptr;
    }
}

}
