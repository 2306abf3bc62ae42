// Kernel generation: turns one fusion group into CUDA C++ source that
// instantiates the hand-written skeleton building blocks (skeleton/*.cuh), plus
// the launch plan the executor needs (argument layout, tiles, TMA boxes).
//
// This replaces the reference's OpenCL code generators (runtime/skeleton/*.cpp):
// the per-cell expression of the group is emitted as straight-line code with
// canonical (position-based) names, so groups with equal structure produce
// identical source and share one compiled module, as the reference's Version
// cache shares one program per signature (runtime/Program.cpp:64).
#pragma once

#include "fusion.hpp"

#include <string>
#include <vector>

namespace mapb {

struct TmaSpec {
  int in_index = 0;     // index into the plan's raster inputs
  int dtype = 0;
  int box_w = 0, box_h = 0;
  int pad_x = 0;        // tile column 0 is raster column (x0 - pad_x)
  int halo_y = 0;
  size_t smem_off = 0;  // offset of the staged tile in dynamic shared memory
};

// Tile shape of the Local / Focal / Zonal skeletons: TW x TH cells per CTA of NT threads.
struct TileCfg {
  int tw = 64, th = 32, nt = 256;
  int minb = 0;   // focal kernels: minimum resident CTAs per SM in the launch bounds (0: none)
  // focal kernels of the executor's own launches: interior tiles may store a
  // single output with one TMA tile store (FocalTune::tstore says for which
  // groups); the batched and serving dispatchers keep per-cell stores
  bool tile_store = false;
};
bool tile_cfg_valid(const TileCfg &c);
// Whether a focal group's interior tiles compute four byte cells of a row per
// thread step (packed 16-bit lanes; integer bodies on byte rasters).
bool focal_quad_form(const Group &g);
// Whether a focal group holds a hillshade composition in the fast rewritten form.
bool focal_fast_shade(const Group &g);

struct KernelPlan {
  int skeleton = SK_LOCAL;
  std::string source;
  std::string body;         // group code without include and kernel wrapper (Local / Focal), for batching
  size_t bar_off = 0;       // Focal: offset of the TMA mbarrier in dynamic shared memory
  std::string kname;        // main kernel
  std::string kname_final;  // zonal finalisation kernel (empty otherwise)
  size_t args_size = 0;
  // argument layout (byte offsets inside the kernel's argument struct)
  size_t off_tm = 0, off_in = 0, off_out = 0, off_s = 0, off_geom = 0, off_err = 0, off_part = 0, off_aux = 0;
  size_t final_args_size = 0;
  std::vector<Node *> in_rasters;   // a.in[k]
  std::vector<Node *> out_rasters;  // a.out[k]
  std::vector<Node *> scalars;      // a.s[k]
  std::vector<Node *> zonal;        // reductions, in partial-slot order
  std::vector<TmaSpec> tma;
  // Output tile stores (focal, opt-in): in_index is the output's index, the
  // staging tile sits at smem_off, the tensor maps follow the inputs' maps.
  std::vector<TmaSpec> tma_out;
  int threads = 256;
  int tile_w = 64, tile_h = 32;
  int min_blocks = 0;   // minimum resident CTAs per SM in the launch bounds (0: none)
  bool tile_store = false;   // TileCfg::tile_store
  int halo_x = 0, halo_y = 0;
  size_t smem_bytes = 0;
  int aux_count = 0;
  // radial / spreading specifics
  Node *core = nullptr;
};

KernelPlan generate_kernel(const Group &g, TileCfg cfg = TileCfg());

// Tuning overrides of the standalone Local / Focal skeletons, read once from the
// environment variable MAP_B200_FOCAL_TUNE ("key=value,..."; the keys are the
// field names below; absent = the built-in choice, which the measured defaults
// in executor.cpp set). Used to measure variants: every variant computes the
// same cells with the same operations, so results are identical.
struct FocalTune {
  int unroll = 0;   // unroll factor of the per-thread row loop (0: by body weight)
  int defer = 1;    // interior tiles keep a thread's results in registers and store them last
  int nt = 0, tw = 0, th = 0;
  int lnt = 0, ltw = 0, lth = 0;   // the same for standalone Local kernels
  int qnt = 0, qtw = 0, qth = 0;   // the same for focal kernels of the packed byte form
  int minb = 0;                     // focal kernels: minimum resident CTAs per SM (register cap)
  int pdl = 1;                      // Local / Focal kernels as programmatic dependent launches (0: plain launches)
  int fpair = 0;                    // the fast hillshade form in the paired (f32x2) form as well
  int cpair = 0;                    // pairs of cells (x, x + 1) of one row instead of (y, y + 1) of one column
  int fflag = 0;                    // fast form's non-finite record: comparison (0) or unsigned maximum (1, measured
                                    // 2.5% slower: a dependent chain through the record)
  int fmerge = 1;                   // fast form: the exact leading term of a derivative sum as the addend of the
                                    // neighbouring fused multiply-add (0: every sum from +0)
  int tstore = 1;                   // interior tiles store a single output through shared memory with one TMA
                                    // tile store instead of one global store per cell: 1 for the fast hillshade
                                    // form (558 against 535 Gcells/s), 2 for every single-output focal group, 0 off
};
const FocalTune &focal_tune();

// Dynamic shared memory of a radial scan launch over a W x H raster: two front
// buffers when they fit (0 otherwise: the kernel then re-reads fronts from its output).
size_t radial_front_smem(int W, int H, int dtype);
// Pointer-jumping flow accumulation (integer types): cell limit, rounds for N
// cells, whether a type qualifies, and the scratch bytes for N cells.
size_t spread_pj_cells();
int spread_pj_rounds(size_t N);
bool spread_pj_type(int dt);
size_t spread_pj_scratch(size_t N, int dt);

// Reference float-constant rounding: constants written into kernel text by the
// reference go through std::to_string ("%f", six decimals) before the device
// compiler parses them (util/VariantType.cpp:89-104, runtime/skeleton/util.cpp mask_decl).
Variant reference_literal_value(const Variant &v);

}  // namespace mapb
