// Inverse-Hopf product grids on SO(3)/K (src/hopf.zig): the reference's default sample
// generator, built on the host in FP64 and rounded once to f32 rows, which the engine then
// folds into the zone on the GPU.
#pragma once
#include <cstdint>
#include <optional>
#include <vector>

namespace zo::hopf {

constexpr uint32_t kMaxFrequency = 512;     // src/hopf.zig:22
constexpr uint64_t kMaxCount = 10000000;    // src/hopf.zig:23

// Root grid of a group (I wherever the group embeds in I, else O or D6); group ids are the
// engine's (C2 C3 C4 C6 D2 D3 D4 D6 T O I = 0..10).
int root_of(int gid);
// Orientations of the frequency-f grid (fibre count x node count / |K|), unchecked.
uint64_t raw_count(int gid, uint32_t f);
// The same, checked: throws on f outside 1..512 (InvalidGridResolution) or a count above
// ten million (GridTooLarge).
uint32_t count(int gid, uint32_t f);
// Frequency whose count is nearest `target` by ratio (src/hopf.zig:86-99).
uint32_t nearest_frequency(int gid, uint32_t target);
// Frequency with the largest count not above `budget` (src/hopf.zig:101-113).
std::optional<uint32_t> largest_frequency(int gid, uint32_t budget);
// The grid's rows, 4 floats each (w, x, y, z), one orbit image per orientation, in the
// reference's row order (src/hopf.zig:528-607). Throws on an invalid frequency.
std::vector<float> points(int gid, uint32_t f);
// Generator name shown in the stats (src/engine.zig:271-275).
const char* generator_name(int gid);

}  // namespace zo::hopf
