// star_special.cu — kernel variants specialised for the common query shapes
// (filters, bitmap-decided probes, table probes), in their own translation unit so the
// build compiles them in parallel with the generic variants.
#include "star_impl.cuh"

namespace mb {

#define MB_SHAPE_VARIANTS(NF, ND, NS)                                                                  \
  {4, 16, NF, ND, NS, star_kernel<4, 16, NF, ND, NS>}, {8, 8, NF, ND, NS, star_kernel<8, 8, NF, ND, NS>}, \
      {16, 8, NF, ND, NS, star_kernel<16, 8, NF, ND, NS>}, {8, 16, NF, ND, NS, star_kernel<8, 16, NF, ND, NS>}

// the same shapes packing the first sparse probe's survivors across the warp before the
// second round (used where the tuned configuration asks for it)
#define MB_PACK_VARIANTS(NF, ND, NS)                                                                \
  {8, 8, NF, ND, NS, star_kernel<8, 8, NF, ND, NS, false, true>, false, true},                      \
      {16, 8, NF, ND, NS, star_kernel<16, 8, NF, ND, NS, false, true>, false, true},                \
      {8, 16, NF, ND, NS, star_kernel<8, 16, NF, ND, NS, false, true>, false, true}

// the packed shapes that return each stage to the producer before the last batch's probes
#define MB_REL_VARIANTS(NF, ND, NS)                                                                   \
  {8, 8, NF, ND, NS, star_kernel<8, 8, NF, ND, NS, false, true, true>, false, true, true},            \
      {16, 8, NF, ND, NS, star_kernel<16, 8, NF, ND, NS, false, true, true>, false, true, true}

// the same shapes reading cluster-resident mirrors in the sparse phase
#define MB_MIRROR_VARIANTS(NF, ND, NS)                                                        \
  {8, 8, NF, ND, NS, star_kernel<8, 8, NF, ND, NS, true>, true},                              \
      {16, 8, NF, ND, NS, star_kernel<16, 8, NF, ND, NS, true>, true},                        \
      {8, 16, NF, ND, NS, star_kernel<8, 16, NF, ND, NS, true>, true}

static const Variant kSpecial[] = {
    MB_SHAPE_VARIANTS(3, 0, 0),  // filter-aggregate (q11.cu)
    MB_SHAPE_VARIANTS(0, 1, 2),  // Query A: supplier bitmap, part and date tables (q21.cu)
    MB_SHAPE_VARIANTS(0, 1, 3),  // Query B: supplier bitmap, customer, part, date (q41.cu)
    MB_SHAPE_VARIANTS(2, 1, 4),  // engine filter_probe_group_by: supplier bitmap, four tables
    MB_SHAPE_VARIANTS(0, 1, 4),  // engine probe_group_by: supplier bitmap, four tables
    MB_SHAPE_VARIANTS(0, 0, 1),  // src/ops probe, one table
    MB_PACK_VARIANTS(0, 1, 3),
    MB_PACK_VARIANTS(2, 1, 4),
    MB_PACK_VARIANTS(0, 1, 4),
    MB_REL_VARIANTS(0, 1, 3),
    MB_REL_VARIANTS(2, 1, 4),
    MB_REL_VARIANTS(0, 1, 4),
    MB_MIRROR_VARIANTS(0, 1, 2),
    MB_MIRROR_VARIANTS(0, 1, 3),
    MB_MIRROR_VARIANTS(2, 1, 4),
    MB_MIRROR_VARIANTS(0, 1, 4),
};

const Variant* star_variants_special(int* count) {
  *count = static_cast<int>(sizeof(kSpecial) / sizeof(kSpecial[0]));
  return kSpecial;
}

}  // namespace mb
