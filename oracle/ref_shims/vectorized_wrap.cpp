// Compiles the reference's cpu/vectorized.cpp unmodified, except that its definition of
// Primitives::ordaggr_count is renamed out of the way: that function falls off its end without
// a return (cpu/vectorized.cpp:649-656), which GCC 13 turns into a trap at any optimisation
// level. ref_bridge.cpp supplies a definition of ordaggr_count with the same behaviour
// (count += lim[g] - previous lim) that returns.
#define ordaggr_count ordaggr_count_without_return_unused
#include "vectorized.cpp"
#undef ordaggr_count
