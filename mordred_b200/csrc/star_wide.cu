// star_wide.cu — kernel variants with more consumer warps than tile slices: 20 or 24 warps
// over 16 slices of 256 rows (28 measured no faster than 24). A warp copies its last
// batch's columns into registers and returns the stage before it probes, so the extra
// warps probe the survivors of earlier slices while others run the dense phase of later
// ones. In a translation unit of their own so the build compiles them in parallel.
#include "star_impl.cuh"

namespace mb {

#define MB_WIDE_VARIANTS(NF, ND, NS)                                                                     \
  {20, 8, NF, ND, NS, star_kernel<20, 8, NF, ND, NS, false, true, false>, false, true, false},           \
      {24, 8, NF, ND, NS, star_kernel<24, 8, NF, ND, NS, false, true, false>, false, true, false},       \
      {20, 8, NF, ND, NS, star_kernel<20, 8, NF, ND, NS, false, true, true>, false, true, true},         \
      {24, 8, NF, ND, NS, star_kernel<24, 8, NF, ND, NS, false, true, true>, false, true, true}

// unpacked, returning each stage early (the Query A shape: its second round is one small table)
#define MB_WIDE_PLAIN_VARIANTS(NF, ND, NS)                                                               \
  {20, 8, NF, ND, NS, star_kernel<20, 8, NF, ND, NS, false, false, true>, false, false, true},           \
      {24, 8, NF, ND, NS, star_kernel<24, 8, NF, ND, NS, false, false, true>, false, false, true}

static const Variant kWide[] = {
    MB_WIDE_PLAIN_VARIANTS(0, 1, 2),  // Query A
    MB_WIDE_VARIANTS(0, 1, 3),  // Query B
    MB_WIDE_VARIANTS(2, 1, 4),  // engine filter_probe_group_by
    MB_WIDE_VARIANTS(0, 1, 4),  // engine probe_group_by
};

const Variant* star_variants_wide(int* count) {
  *count = static_cast<int>(sizeof(kWide) / sizeof(kWide[0]));
  return kWide;
}

}  // namespace mb
