// C ABI and host orchestration of the B200 descriptor / GAP path.
//
// Host objects mirror the reference's: a calculator owns its hypers and the
// radial spline (calculator_spherical_expansion.hh:1019-1156), a structure set
// owns the structures, their neighbour list and the computed features
// (ManagerCollection + Properties, structure_manager_collection.hh), a GAP
// model owns the sparse points and weights (models/krr.py, sparse_points.hh).
// Every device buffer is owned by one of these handles and reused across
// calls; kernels run on the structure set's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "common.cuh"
#include "json_lite.h"

namespace rgpu {
int64_t launches(bool reset);
extern bool g_tf32_split;
}  // namespace rgpu

using namespace rgpu;

namespace {

thread_local std::string t_err;
thread_local int t_kind = RGPU_EXC_NONE;

int fail(const Error & e) {
  t_err = e.what();
  t_kind = e.kind;
  return e.code;
}

template <class F>
int guard(F && f) {
  try {
    t_err.clear();
    t_kind = RGPU_EXC_NONE;
    f();
    return RGPU_OK;
  } catch (const Error & e) {
    return fail(e);
  } catch (const std::bad_alloc &) {
    return fail(Error(RGPU_ERR_CUDA, "host allocation failed"));
  } catch (const std::exception & e) {
    return fail(Error(RGPU_ERR_INVALID_ARGUMENT, e.what()));
  }
}

const double kPi = 3.14159265358979323846264338327950288;

}  // namespace

// ------------------------------------------------------------------- hypers
namespace rgpu {
void parse_hypers(const std::string & kind, const std::string & text, Hypers & h) {
  Json j = Json::parse(text);
  if (j.type != Json::Object) throw Error(RGPU_ERR_INVALID_ARGUMENT, "hypers must be a JSON object");
  h.kind = kind;
  if (kind != "sphericalinvariants" && kind != "sphericalexpansion")
    throw Error(RGPU_ERR_INVALID_ARGUMENT,
                "The representations factory " + kind +
                    " has not been registered. The available combinations are: "
                    "['sphericalexpansion', 'sphericalinvariants']");
  h.max_radial = j.at("max_radial").as_int();
  h.max_angular = j.at("max_angular").as_int();
  if (h.max_radial < 1) throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_radial must be >= 1");
  if (h.max_angular < 0 || h.max_angular > kMaxL)
    throw Error(RGPU_ERR_INVALID_ARGUMENT, "max_angular must be in [0, 12] on the GPU path");
  h.compute_gradients = j.has("compute_gradients") ? j.at("compute_gradients").as_bool() : false;
  if (kind == "sphericalinvariants") {
    h.normalize = j.at("normalize").as_bool();
    h.soap_type = j.at("soap_type").as_string();
    if (h.soap_type != "PowerSpectrum") {
      if (h.soap_type == "RadialSpectrum" || h.soap_type == "BiSpectrum")
        throw Error(RGPU_ERR_INVALID_ARGUMENT,
                    "Requested SphericalInvariants type '" + h.soap_type +
                        "' is not on the B200 path. Supported: 'PowerSpectrum'.");
      throw Error(RGPU_ERR_INVALID_ARGUMENT,
                  "Requested SphericalInvariants type '" + h.soap_type +
                      "' has not been implemented.  Must be one of: 'PowerSpectrum', "
                      "'RadialSpectrum', or 'BiSpectrum'.");
    }
    if (j.has("coefficient_subselection"))
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "coefficient_subselection is not on the B200 path");
  }
  if (j.has("expansion_by_species_method")) {
    std::string m = j.at("expansion_by_species_method").as_string();
    if (m != "environment wise" && m != "user defined" && m != "structure wise")
      throw Error(RGPU_ERR_INVALID_ARGUMENT,
                  "expansion_by_species_method provided:'" + m +
                      "' is not part of the implemented methods: 'environment wise', "
                      "'structure wise', 'user defined', ");
  }
  const Json & fc = j.at("cutoff_function");
  std::string fct = fc.at("type").as_string();
  if (fct != "ShiftedCosine" && fct != "RadialScaling")
    throw Error(RGPU_ERR_INVALID_ARGUMENT,
                "Requested cutoff function type '" + fct + "' is not on the B200 path. Supported: "
                                                          "'ShiftedCosine', 'RadialScaling'.");
  h.cutoff = fc.at("cutoff").at("value").as_number();
  h.smooth_width = fc.at("smooth_width").at("value").as_number();
  h.radial_scaling = fct == "RadialScaling";
  if (h.radial_scaling) {
    // representations/cutoff_functions.hh:243-253
    h.rs_rate = fc.at("rate").at("value").as_number();
    if (h.rs_rate < 0) throw Error(RGPU_ERR_INVALID_ARGUMENT, "RadialScaling's rate should be positive");
    h.rs_exponent = fc.at("exponent").at("value").as_number();
    h.rs_scale = fc.at("scale").at("value").as_number();
  }
  const Json & gd = j.at("gaussian_density");
  std::string gt = gd.at("type").as_string();
  if (gt != "Constant")
    throw Error(RGPU_ERR_INVALID_ARGUMENT,
                "Requested Smearing type '" + gt + "' has not been implemented.  Must be one of: 'Constant'.");
  h.sigma = gd.at("gaussian_sigma").at("value").as_number();
  const Json & rc = j.at("radial_contribution");
  std::string rt = rc.at("type").as_string();
  if (rt != "GTO")
    throw Error(RGPU_ERR_INVALID_ARGUMENT,
                "Requested Radial contribution type '" + rt + "' is not on the B200 path. Supported: 'GTO'.");
  h.spline = false;
  h.spline_accuracy = 1e-13;  // direct 1F1 evaluation is served by a spline this fine
  if (rc.has("optimization")) {
    const Json & o = rc.at("optimization");
    if (o.has("RadialDimReduction"))
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "RadialDimReduction is not on the B200 path");
    if (o.has("Spline")) {
      h.spline = true;
      const Json & sp = o.at("Spline");
      if (!sp.has("accuracy")) throw Error(RGPU_ERR_INVALID_ARGUMENT, "No Spline accuracy was given.");
      h.spline_accuracy = sp.at("accuracy").as_number();
      if (!(h.spline_accuracy > 0)) throw Error(RGPU_ERR_INVALID_ARGUMENT, "Error bound must be > 0");
    }
  }
  if (!(h.cutoff > 0)) throw Error(RGPU_ERR_INVALID_ARGUMENT, "cutoff must be > 0");
  h.name = kind + "_" + j.dump();
}
}  // namespace rgpu

// ------------------------------------------------------------------ handles
struct rgpu_calculator {
  int device{-1};  // device of the uploaded tables (-1: not uploaded yet)
  Hypers hy;
  RadialSpline spline;
  DevBuf grid, y, y2h, yf, y2hf, q4f, center;
  SplineDev dev{};
};

struct GapLayout;

// One FP32 prediction (rgpu_gap_predict / rgpu_gap_predict_stress) recorded
// as a CUDA graph for one size bucket: the same model, output kind, numbers
// of structures and atoms, species layout and centres per species, and the
// same device buffers; the neighbour list inside is built to capacities
// 12.5 % above the counts of the recording call.
struct PredictGraph {
  cudaGraph_t graph{nullptr};
  cudaGraphExec_t exec{nullptr};
  const rgpu_gap_model * model{nullptr};
  bool stress{false}, outputs{false};
  int n_struct{0};
  int64_t n_atoms{0};
  std::vector<int> species;
  std::vector<int64_t> species_count;
  NlCaps caps{};
  std::vector<const void *> buffers;
  double * out_h{nullptr};  // pinned: energies, forces, stress sums of a replay
  int64_t kernels{0};
  uint64_t used{0};
};

struct rgpu_structures {
  int device{-1};  // device current at creation: owns the stream and every buffer
  cudaStream_t st{nullptr};
  int n_struct{0};
  int64_t n_atoms{0};
  std::vector<int64_t> atom_off;
  std::vector<int32_t> types;
  std::vector<double> cells_h;  // [n_struct][9], lattice vectors as rows
  std::vector<uint8_t> mask;
  bool has_mask{false};
  std::vector<int64_t> center_off_h;
  DevBuf atom_off_d, pos_d, types_d, cells_d, pbc_d, tag2idx_d, ncent_d, center_off_d, atom_struct_d;
  // staging (pinned) for host inputs
  void * pinned{nullptr};
  size_t pinned_cap{0};
  // neighbour list
  bool nl_valid{false};
  double nl_cutoff{-1};
  NlWork nlw;
  NlOutputs nl;
  std::vector<int64_t> pair_off_h;  // host copy of nl.pair_off, made on demand
  bool pair_off_h_valid{false};
  std::vector<int> batch_species;   // sorted atom types present in the batch
  int64_t centres_of_type[130]{};   // centres per atom type (the mask applied)
  // layout and features
  std::vector<int> species;  // dense layout (sorted)
  DevBuf lut;
  FeatureDims fd{};
  std::vector<int64_t> species_count;
  DevBuf row_of_center, center_of_row, species_count_d, sort_tmp, present, tile_mask;
  DevBuf C64, X64, invn64, C32, X32, xscale32;  // xscale32[row] = 1/|p| (FP32 path)
  int feat_precision{-1};
  const rgpu_calculator * feat_calc{nullptr};
  bool feat_gradients{false};
  bool feat_valid{false};
  // GAP work
  DevBuf E_d, F_d, S_d, K64, t64, erow64, Wh, Wl, dX32, dC32, epart, Xh, Xl, chunk_map;
  bool feat_x32{false};  // FP32 features also kept unsplit (for export)
  DevBuf dCp, dCs, dXp;
  DevBuf knm, W64, plist, Vvir;  // sparse kernel matrices for training
  // MD step recorded as a CUDA graph (rgpu_md_step)
  cudaGraph_t md_graph{nullptr};
  cudaGraphExec_t md_exec{nullptr};
  const rgpu_gap_model * md_model{nullptr};
  bool md_stress{false};
  NlCaps md_caps{};
  std::vector<const void *> md_buffers;  // device buffer addresses at recording
  std::vector<int> md_species;
  int64_t md_replays{0};       // replays since the graph was recorded
  int64_t md_kernels{0};       // kernel nodes of the recorded graph
  int64_t md_reason{0};        // why the last step did not replay: 0 none (first step or no
                               // recording), 1 a buffer moved, 3 model or layout, 100 + status
  bool md_no_graph{false};     // recording failed once: ordinary path only
  double * md_pos_h{nullptr};  // pinned: positions in, outputs out
  double * md_out_h{nullptr};
  size_t md_pos_cap{0}, md_out_cap{0};
  // FP32 predictions recorded as CUDA graphs, a few size buckets per handle
  std::vector<PredictGraph> pgraphs;
  bool use_graphs{true};
  uint64_t pgraph_clock{0};
  int64_t pgraph_replays{0}, pgraph_records{0}, pgraph_last_kernels{0};
  // autograd: the model whose forward (rgpu_gap_forward_dev) left W, the
  // features and the list in place for rgpu_gap_backward_dev (null: none)
  const rgpu_gap_model * fwd_model{nullptr};
  DevBuf y0_d;  // per-structure energy baseline of fwd_model
  // status and timing
  DevStatus * status_d{nullptr};
  DevStatus * status_h{nullptr};
  cudaEvent_t ev[10]{};
  double stage_ms[10]{};
  bool timed{false};
};

struct rgpu_gap_model {
  int device{-1};  // device of the model's buffers (-1: none allocated yet)
  rgpu_calculator * calc{nullptr};
  std::vector<int> species;  // model layout species (sorted)
  int M{0};
  std::vector<int32_t> sp_species;
  std::vector<double> T;  // M x D_model
  std::vector<double> alpha;
  int zeta{2};
  std::vector<double> self_contrib;  // per model species
  // device copies for a batch layout
  std::vector<int> layout_species;
  int layout_D{0};
  std::vector<GapSpecies> segs;  // per batch species
  DevBuf T64, alpha64, Th, Tl, Tth, Ttl, alpha32;
  std::vector<int64_t> tt_off;  // per batch species offset into Tt32
  DevBuf ucol;                  // caller's index of each sparse point in layout order
  std::vector<double> T_layout, alpha_layout;  // host copies in the batch layout
  int64_t tt_total{0};
  bool layout_bf16{false};
};

namespace {

// Runs the rest of a call on a structure set's device and gives the caller
// back the device that was current before. A structure set belongs to the
// device that was current when it was created (its stream and buffers live
// there), so a call made while another device is current still works on its
// own device's memory.
struct OnDevice {
  int prev{-1};
  explicit OnDevice(const rgpu_structures * s) {
    if (!s || s->device < 0) return;
    int cur = 0;
    RGPU_CUDA(cudaGetDevice(&cur));
    if (cur != s->device) {
      RGPU_CUDA(cudaSetDevice(s->device));
      prev = cur;
    }
  }
  ~OnDevice() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  OnDevice(const OnDevice &) = delete;
  OnDevice & operator=(const OnDevice &) = delete;
};

// Ties a calculator or model to the current device on its first device
// allocation, and rejects later use with a structure set of another device
// (its buffers would be another GPU's memory).
void bind_device(int & owner, const char * what) {
  const int dev = current_device();
  if (owner < 0) {
    owner = dev;
  } else if (owner != dev) {
    throw Error(RGPU_ERR_INVALID_ARGUMENT, std::string(what) + " lives on device " + std::to_string(owner) +
                                               " and cannot be used with a structure set of device " +
                                               std::to_string(dev));
  }
}

void ensure_stream(rgpu_structures * s) {
  if (!s->st) {
    s->device = current_device();
    RGPU_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
    RGPU_CUDA(cudaMalloc(&s->status_d, sizeof(DevStatus)));
    RGPU_CUDA(cudaMemset(s->status_d, 0, sizeof(DevStatus)));
    RGPU_CUDA(cudaMallocHost(&s->status_h, sizeof(DevStatus)));
    for (auto & e : s->ev) RGPU_CUDA(cudaEventCreate(&e));
  }
}

void * staging(rgpu_structures * s, size_t bytes) {
  if (bytes > s->pinned_cap) {
    if (s->pinned) {
      RGPU_CUDA(cudaStreamSynchronize(s->st));  // no copy in flight may still use it
      cudaFreeHost(s->pinned);
    }
    s->pinned = nullptr;
    RGPU_CUDA(cudaMallocHost(&s->pinned, bytes));
    s->pinned_cap = bytes;
  }
  return s->pinned;
}

// Host -> device through the pinned staging buffer, in order on the stream.
void upload(rgpu_structures * s, DevBuf & dst, const void * src, size_t bytes) {
  dst.ensure(bytes);
  if (bytes == 0) return;
  RGPU_CUDA(cudaStreamSynchronize(s->st));  // staging buffer reuse
  void * p = staging(s, bytes);
  std::memcpy(p, src, bytes);
  RGPU_CUDA(cudaMemcpyAsync(dst.p, p, bytes, cudaMemcpyHostToDevice, s->st));
}

// Several host -> device copies through one pass of the staging buffer: a
// single wait for the previous use of the buffer, then one copy per array.
struct Upload {
  DevBuf * dst;
  const void * src;
  size_t bytes;
};
void upload_many(rgpu_structures * s, const std::vector<Upload> & ups) {
  size_t total = 0;
  for (const Upload & u : ups) total += (u.bytes + 255) & ~size_t(255);
  for (const Upload & u : ups) u.dst->ensure(u.bytes);
  if (total == 0) return;
  RGPU_CUDA(cudaStreamSynchronize(s->st));  // staging buffer reuse
  unsigned char * base = static_cast<unsigned char *>(staging(s, total));
  size_t off = 0;
  for (const Upload & u : ups) {
    if (u.bytes == 0) continue;
    std::memcpy(base + off, u.src, u.bytes);
    RGPU_CUDA(cudaMemcpyAsync(u.dst->p, base + off, u.bytes, cudaMemcpyHostToDevice, s->st));
    off += (u.bytes + 255) & ~size_t(255);
  }
}

void mark(rgpu_structures * s, int i) {
  if (s->timed) RGPU_CUDA(cudaEventRecord(s->ev[i], s->st));
}

FeatureDims make_dims(const Hypers & hy, int S) {
  FeatureDims f;
  f.S = S;
  f.n = hy.max_radial;
  f.L = hy.max_angular;
  f.K = (f.L + 1) * (f.L + 1);
  f.W = f.n * (f.L + 1);
  f.nK = f.n * f.K;
  f.P = S * (S + 1) / 2;
  f.D = f.P * f.n * f.n * (f.L + 1);
  f.Dpad = (f.D + 31) / 32 * 32;
  f.Sn = S * f.n;
  if (f.n % 2 == 0) {  // row pairs never straddle two species
    f.G = S;
    f.npg = f.n / 2;
  } else {
    f.G = 1;
    f.npg = (f.Sn + 1) / 2;
  }
  f.TD = f.npg * (f.npg + 1) / 2;
  f.TO = f.npg * f.npg;
  f.lenD = (4 * (f.L + 1) * f.TD + 31) / 32 * 32;
  f.lenO = (4 * (f.L + 1) * f.TO + 31) / 32 * 32;
  f.Dg = f.G * f.lenD + f.G * (f.G - 1) / 2 * f.lenO;
  return f;
}

// Choose the dense species layout: batch species plus `extra`.
void set_layout(rgpu_structures * s, const Hypers & hy, const std::vector<int> & extra) {
  std::set<int> sp(s->batch_species.begin(), s->batch_species.end());
  sp.insert(extra.begin(), extra.end());
  std::vector<int> species(sp.begin(), sp.end());
  if (int(species.size()) > kMaxSpecies)
    throw Error(RGPU_ERR_INVALID_ARGUMENT, "more than 16 species in one batch is not supported on the GPU");
  FeatureDims fd = make_dims(hy, int(species.size()));
  bool same = species == s->species && fd.n == s->fd.n && fd.L == s->fd.L;
  s->fd = fd;
  if (same) return;
  s->species = species;
  std::vector<int8_t> lut(130, -1);
  for (size_t i = 0; i < species.size(); ++i) lut[species[i]] = int8_t(i);
  upload(s, s->lut, lut.data(), lut.size());
  s->feat_valid = false;
}

void build_nl(rgpu_structures * s, double cutoff) {
  if (s->nl_valid && s->nl_cutoff == cutoff) return;
  s->fwd_model = nullptr;
  NlInputs in;
  in.n_struct = s->n_struct;
  in.n_atoms = s->n_atoms;
  in.atom_off = s->atom_off_d.as<int64_t>();
  in.pos = s->pos_d.as<double>();
  in.types = s->types_d.as<int32_t>();
  in.cells = s->cells_d.as<double>();
  in.pbc = s->pbc_d.as<int32_t>();
  in.tag2idx = s->has_mask ? s->tag2idx_d.as<int32_t>() : nullptr;
  in.n_centers = s->ncent_d.as<int32_t>();
  in.center_off = s->center_off_d.as<int64_t>();
  in.atom_struct = s->atom_struct_d.as<int32_t>();
  in.n_centers_total = s->center_off_h[s->n_struct];
  build_neighbour_list(in, cutoff, s->nlw, s->nl, s->status_d, s->status_h, s->st);
  s->pair_off_h_valid = false;
  s->nl_valid = true;
  s->nl_cutoff = cutoff;
  s->feat_valid = false;
}

// Host copy of the neighbour list's centre offsets (for chunking the plain
// path's gradient passes).
const std::vector<int64_t> & pair_offsets_host(rgpu_structures * s) {
  if (!s->pair_off_h_valid) {
    s->pair_off_h.resize(s->nl.n_centers + 1);
    RGPU_CUDA(cudaMemcpyAsync(s->pair_off_h.data(), s->nl.pair_off, sizeof(int64_t) * (s->nl.n_centers + 1),
                              cudaMemcpyDeviceToHost, s->st));
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    s->pair_off_h_valid = true;
  }
  return s->pair_off_h;
}

ExpansionArgs exp_args(const rgpu_calculator * c, const rgpu_structures * s) {
  ExpansionArgs a;
  a.fd = s->fd;
  a.sp = c->dev;
  a.center_contrib = c->center.as<double>();
  a.species_lut = s->lut.as<int8_t>();
  a.rc = c->hy.cutoff;
  a.sw = c->hy.smooth_width;
  a.rs.on = c->hy.radial_scaling ? 1 : 0;
  a.rs.rate = c->hy.rs_rate;
  a.rs.exponent = c->hy.rs_exponent;
  a.rs.scale = c->hy.rs_scale;
  a.n_centers = s->nl.n_centers;
  a.center_atom = s->nl.center_atom;
  a.pair_off = s->nl.pair_off;
  a.pair_j = s->nl.pair_j;
  a.pair_dist = s->nl.pair_dist;
  a.pair_dir = s->nl.pair_dir;
  a.types = s->types_d.as<int32_t>();
  return a;
}

// Species sort of the centres: row order of X (grouped by central species).
void sort_rows(rgpu_structures * s) {
  const int64_t nc = s->nl.n_centers;
  s->row_of_center.ensure(sizeof(int32_t) * (nc + 1));
  s->center_of_row.ensure(sizeof(int32_t) * (nc + 1));
  s->species_count_d.ensure(sizeof(int64_t) * kMaxSpecies);
  launch_species_sort(nc, s->types_d.as<int32_t>(), s->nl.center_atom, s->lut.as<int8_t>(), s->fd.S,
                      s->species_count_d.as<int64_t>(), s->row_of_center.as<int32_t>(),
                      s->center_of_row.as<int32_t>(), s->sort_tmp, s->st);
  // the counts per central species are known on the host since the upload
  s->species_count.assign(s->fd.S, 0);
  for (int sI = 0; sI < s->fd.S; ++sI) s->species_count[sI] = s->centres_of_type[s->species[sI]];
}

// After the FP32 expansion (which writes the presence masks): rows of one
// species ordered by their neighbour species, so that the GEMM tiles of the
// packed layout's species segments can skip what none of their rows holds.
// Only layouts with more than one segment group need it.
void sort_rows_by_mask(rgpu_structures * s) {
  if (s->fd.G < 2) return;
  launch_mask_sort(s->nl.n_centers, s->types_d.as<int32_t>(), s->nl.center_atom, s->lut.as<int8_t>(),
                   s->present.as<uint32_t>(), s->fd.S, s->row_of_center.as<int32_t>(), s->center_of_row.as<int32_t>(),
                   s->sort_tmp, s->st);
}

void compute_features(rgpu_calculator * c, rgpu_structures * s, int precision, bool grads,
                      const std::vector<int> & extra_species, bool need_x32 = true) {
  build_nl(s, c->hy.cutoff);
  set_layout(s, c->hy, extra_species);
  if (s->feat_valid && s->feat_calc == c && s->feat_precision == precision &&
      (precision == RGPU_PRECISION_FP64 || s->feat_x32 || !need_x32)) {
    s->feat_gradients = s->feat_gradients || grads;
    return;
  }
  s->fwd_model = nullptr;
  mark(s, 2);
  sort_rows(s);
  const int64_t nc = s->nl.n_centers;
  const FeatureDims & fd = s->fd;
  ExpansionArgs ea = exp_args(c, s);
  s->present.ensure(sizeof(uint32_t) * (nc + 1));
  PsArgs pa;
  pa.fd = fd;
  pa.n_centers = nc;
  pa.normalize = c->hy.normalize;
  pa.row_of_center = s->row_of_center.as<int32_t>();
  if (precision == RGPU_PRECISION_FP64) {
    s->C64.ensure(sizeof(double) * size_t(nc) * fd.S * fd.nK + 64);
    launch_expansion_fp64(ea, s->C64.as<double>(), s->present.as<uint32_t>(), s->st);
    mark(s, 3);
    if (c->hy.kind == "sphericalinvariants") {
      s->X64.ensure(sizeof(double) * size_t(nc) * fd.Dpad + 64);
      s->invn64.ensure(sizeof(double) * (nc + 1));
      launch_ps_fwd_fp64(pa, s->C64.as<double>(), s->X64.as<double>(), s->invn64.as<double>(), s->st);
    }
  } else {
    s->C32.ensure(sizeof(float) * size_t(nc) * fd.S * fd.n * row_stride(fd.L) + 64);
    launch_expansion_fp32(ea, s->C32.as<float>(), s->present.as<uint32_t>(), s->st);
    if (c->hy.kind == "sphericalinvariants") sort_rows_by_mask(s);
    mark(s, 3);
    if (c->hy.kind == "sphericalinvariants") {
      if (need_x32) s->X32.ensure(sizeof(float) * size_t(nc) * fd.Dg + 64);
      s->Xh.ensure(sizeof(uint16_t) * size_t(nc) * fd.Dg + 64);
      s->Xl.ensure(sizeof(uint16_t) * size_t(nc) * fd.Dg + 64);
      s->xscale32.ensure(sizeof(float) * (nc + 1));
      pa.present = s->present.as<uint32_t>();
      launch_ps_fwd_fast(pa, s->C32.as<float>(), need_x32 ? s->X32.as<float>() : nullptr,
                         s->Xh.as<__nv_bfloat16>(), s->Xl.as<__nv_bfloat16>(), s->xscale32.as<float>(), s->st);
    }
    s->feat_x32 = need_x32;
  }
  s->feat_valid = true;
  s->feat_calc = c;
  s->feat_precision = precision;
  s->feat_gradients = grads;
}

// Keys present in the batch, as the reference's union of per-centre keys.
std::vector<std::pair<int, int>> present_keys(const rgpu_calculator * c, const rgpu_structures * s) {
  const int64_t nc = s->nl.n_centers;
  std::vector<uint32_t> pres(nc);
  RGPU_CUDA(cudaMemcpyAsync(pres.data(), s->present.p, sizeof(uint32_t) * nc, cudaMemcpyDeviceToHost, s->st));
  RGPU_CUDA(cudaStreamSynchronize(s->st));
  std::set<uint32_t> masks(pres.begin(), pres.end());
  std::set<std::pair<int, int>> keys;
  for (uint32_t m : masks) {
    for (int a = 0; a < s->fd.S; ++a) {
      if (!(m >> a & 1)) continue;
      if (c->hy.kind == "sphericalexpansion") {
        keys.insert({s->species[a], s->species[a]});
        continue;
      }
      for (int b = a; b < s->fd.S; ++b)
        if (m >> b & 1) keys.insert({s->species[a], s->species[b]});
    }
  }
  return std::vector<std::pair<int, int>>(keys.begin(), keys.end());
}

// Column blocks of the dense layout for the requested keys (-1 = absent).
std::vector<int> key_blocks(const rgpu_calculator * c, const rgpu_structures * s, int n_keys,
                            const int32_t * keys) {
  std::vector<int> blocks(n_keys, -1);
  std::map<int, int> sidx;
  for (int i = 0; i < s->fd.S; ++i) sidx[s->species[i]] = i;
  std::map<std::pair<int, int>, int> kid;
  int k = 0;
  for (int a = 0; a < s->fd.S; ++a)
    for (int b = a; b < s->fd.S; ++b) kid[{a, b}] = k++;
  for (int i = 0; i < n_keys; ++i) {
    int ka = keys[2 * i], kb = keys[2 * i + 1];
    if (!sidx.count(ka)) continue;
    if (c->hy.kind == "sphericalexpansion") {
      blocks[i] = sidx[ka];
      continue;
    }
    if (!sidx.count(kb)) continue;
    int a = sidx[ka], b = sidx[kb];
    if (a > b) std::swap(a, b);
    blocks[i] = kid[{a, b}];
  }
  return blocks;
}

// Dense expansion gradients (property_block_sparse.hh:961-987): 3 rows per
// pair (x, y, z), key blocks of n*K. A pair's gradient has the key of its
// neighbour's species only; the self pair's has every species
// (calculator_spherical_expansion.hh:2327-2366).
void export_expansion_gradient(const rgpu_calculator * calc, rgpu_structures * s, int n_keys,
                               const std::vector<int> & blocks, double * out) {
  const FeatureDims & fd = s->fd;
  const int64_t nc = s->nl.n_centers;
  const int inner = fd.nK;
  ExpansionArgs ea = exp_args(calc, s);
  const std::vector<int64_t> & poff = pair_offsets_host(s);
  const size_t per_pair = sizeof(double) * 3 * size_t(fd.nK);
  const size_t per_center = sizeof(double) * size_t(fd.S) * 3 * fd.nK;
  const size_t budget = size_t(4) << 30;
  std::map<int, int> sidx;
  for (int i = 0; i < fd.S; ++i) sidx[s->species[i]] = i;
  std::vector<double> hp, hs;
  std::vector<int32_t> pj;
  int64_t c0 = 0;
  while (c0 < nc) {
    int64_t c1 = c0;
    size_t bytes = 0;
    while (c1 < nc) {
      size_t add = per_pair * size_t(poff[c1 + 1] - poff[c1]) + per_center;
      if (c1 > c0 && bytes + add > budget) break;
      bytes += add;
      ++c1;
    }
    const int64_t p_base = poff[c0];
    const int64_t np = poff[c1] - p_base;
    s->dCp.ensure(per_pair * size_t(np) + 64);
    s->dCs.ensure(per_center * size_t(c1 - c0) + 64);
    launch_expansion_grad_fp64(ea, c0, c1, p_base, s->dCp.as<double>(), s->st);
    launch_expansion_selfgrad_fp64(ea, c0, c1, p_base, s->dCp.as<double>(), s->dCs.as<double>(), s->st);
    hp.resize(size_t(np) * 3 * fd.nK);
    hs.resize(size_t(c1 - c0) * fd.S * 3 * fd.nK);
    pj.resize(size_t(np));
    RGPU_CUDA(cudaMemcpyAsync(hp.data(), s->dCp.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, s->st));
    RGPU_CUDA(cudaMemcpyAsync(hs.data(), s->dCs.p, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, s->st));
    RGPU_CUDA(cudaMemcpyAsync(pj.data(), s->nl.pair_j + p_base, sizeof(int32_t) * np, cudaMemcpyDeviceToHost,
                              s->st));
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    for (int64_t ci = c0; ci < c1; ++ci)
      for (int64_t p = poff[ci]; p < poff[ci + 1]; ++p) {
        const bool self = (p == poff[ci]);
        const int sj = self ? -1 : sidx.at(s->types[pj[size_t(p - p_base)]]);
        for (int c = 0; c < 3; ++c) {
          double * dst = out + (size_t(p) * 3 + c) * size_t(n_keys) * inner;
          for (int k = 0; k < n_keys; ++k) {
            const int b = blocks[k];
            const double * src = nullptr;
            if (b >= 0 && self)
              src = &hs[((size_t(ci - c0) * fd.S + b) * 3 + c) * fd.nK];
            else if (b >= 0 && b == sj)
              src = &hp[(size_t(p - p_base) * 3 + c) * fd.nK];
            if (src)
              std::memcpy(dst + size_t(k) * inner, src, sizeof(double) * inner);
            else
              std::memset(dst + size_t(k) * inner, 0, sizeof(double) * inner);
          }
        }
      }
    c0 = c1;
  }
}

void model_layout_bf16(rgpu_gap_model * m, rgpu_structures * s);

// Device copies of a model's sparse points in the batch's layout: FP64
// always, the BF16 splits of the tensor-core path only when `bf16` asks.
void model_layout(rgpu_gap_model * m, rgpu_structures * s, bool bf16) {
  bind_device(m->device, "the GAP model");
  const FeatureDims & fd = s->fd;
  if (m->layout_species == s->species && m->layout_D == fd.D) {
    if (bf16 && !m->layout_bf16) model_layout_bf16(m, s);
    return;
  }
  const int Sm = int(m->species.size());
  FeatureDims fm = make_dims(m->calc->hy, Sm);
  std::map<int, int> bidx;
  for (int i = 0; i < fd.S; ++i) bidx[s->species[i]] = i;
  std::vector<std::vector<int>> kb(fd.S, std::vector<int>(fd.S, -1));
  int k = 0;
  for (int a = 0; a < fd.S; ++a)
    for (int b = a; b < fd.S; ++b) kb[a][b] = k++;
  const int blk = fd.n * fd.n * (fd.L + 1);
  // group sparse points by batch species, keep their order inside a species
  std::vector<std::vector<int>> rows(fd.S);
  for (int i = 0; i < m->M; ++i) rows[bidx.at(m->sp_species[i])].push_back(i);
  m->segs.assign(fd.S, GapSpecies{});
  std::vector<double> T(size_t(m->M) * fd.Dpad, 0.), al(m->M);
  int pos = 0;
  int64_t tt_total = 0;
  std::vector<int32_t> user(size_t(std::max(m->M, 1)), 0);
  m->tt_off.assign(fd.S, 0);
  for (int sI = 0; sI < fd.S; ++sI) {
    GapSpecies & g = m->segs[sI];
    g.m0 = pos;
    g.M = int(rows[sI].size());
    g.Mpad = (g.M + 31) / 32 * 32;
    m->tt_off[sI] = tt_total;
    tt_total += int64_t(g.Mpad) * fd.Dg;
    for (int r : rows[sI]) {
      user[pos] = r;
      al[pos] = m->alpha[r];
      const double * src = &m->T[size_t(r) * fm.D];
      double * dst = &T[size_t(pos) * fd.Dpad];
      int km = 0;
      for (int a = 0; a < Sm; ++a)
        for (int b = a; b < Sm; ++b, ++km) {
          int A = bidx.at(m->species[a]), B = bidx.at(m->species[b]);
          int kk = kb[std::min(A, B)][std::max(A, B)];
          std::memcpy(dst + size_t(kk) * blk, src + size_t(km) * blk, sizeof(double) * blk);
        }
      ++pos;
    }
  }
  upload(s, m->T64, T.data(), sizeof(double) * T.size());
  upload(s, m->alpha64, al.data(), sizeof(double) * al.size());
  upload(s, m->ucol, user.data(), sizeof(int32_t) * user.size());
  RGPU_CUDA(cudaStreamSynchronize(s->st));
  m->T_layout.swap(T);
  m->alpha_layout.swap(al);
  m->tt_total = tt_total;
  m->layout_species = s->species;
  m->layout_D = fd.D;
  m->layout_bf16 = false;
  if (bf16) model_layout_bf16(m, s);
}

// BF16 hi/lo splits of T (rows = sparse points) and of T^T per species
// (rows = feature index, padded to Mpad columns) for the tensor-core GEMMs.
void model_layout_bf16(rgpu_gap_model * m, rgpu_structures * s) {
  const FeatureDims & fd = s->fd;
  const std::vector<double> & T = m->T_layout;
  const std::vector<double> & al = m->alpha_layout;
  const int64_t tt_total = m->tt_total;
  auto f2bf = [](float f) -> uint16_t {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0;
    return uint16_t((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
  };
  auto bf2f = [](uint16_t h) -> float {
    uint32_t u = uint32_t(h) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  };
  // the BF16 copies use the packed layout of the FP32 path (padding stays 0)
  std::vector<uint16_t> Th(size_t(std::max(m->M, 1)) * fd.Dg, 0), Tl(Th.size(), 0);
  std::vector<double> packed(fd.Dg);
  for (int r = 0; r < m->M; ++r) {
    pack_reference_row(fd, &T[size_t(r) * fd.Dpad], packed.data());
    for (int d = 0; d < fd.Dg; ++d) {
      const float v = float(packed[d]);
      const size_t o = size_t(r) * fd.Dg + d;
      Th[o] = f2bf(v);
      Tl[o] = f2bf(v - bf2f(Th[o]));
    }
  }
  std::vector<float> al32(al.size());
  for (size_t i = 0; i < al.size(); ++i) al32[i] = float(al[i]);
  std::vector<uint16_t> Tth(size_t(std::max<int64_t>(tt_total, 1)), 0), Ttl(Tth.size(), 0);
  for (int sI = 0; sI < fd.S; ++sI) {
    const GapSpecies & g = m->segs[sI];
    for (int mm = 0; mm < g.M; ++mm)
      for (int d = 0; d < fd.Dg; ++d) {
        const size_t src = size_t(g.m0 + mm) * fd.Dg + d;
        const size_t dst = size_t(m->tt_off[sI]) + size_t(d) * g.Mpad + mm;
        Tth[dst] = Th[src];
        Ttl[dst] = Tl[src];
      }
  }
  upload(s, m->Th, Th.data(), sizeof(uint16_t) * Th.size());
  upload(s, m->Tl, Tl.data(), sizeof(uint16_t) * Tl.size());
  upload(s, m->alpha32, al32.data(), sizeof(float) * al32.size());
  upload(s, m->Tth, Tth.data(), sizeof(uint16_t) * Tth.size());
  upload(s, m->Ttl, Ttl.data(), sizeof(uint16_t) * Ttl.size());
  RGPU_CUDA(cudaStreamSynchronize(s->st));
  m->layout_bf16 = true;
}

size_t plain_budget_bytes() { return size_t(24) << 30; }

void gap_plain(rgpu_gap_model * m, rgpu_structures * s, double * E_d, double * grad_d, bool forces,
               double * stress_d) {
  rgpu_calculator * c = m->calc;
  const FeatureDims & fd = s->fd;
  const int64_t nc = s->nl.n_centers;
  cudaStream_t st = s->st;
  mark(s, 4);
  // forward GEMMs per species: k = X T^T, pointwise, t = W T
  int Mmax = 0;
  for (auto & g : m->segs) Mmax = std::max(Mmax, g.M);
  s->K64.ensure(sizeof(double) * size_t(nc) * std::max(Mmax, 1) + 64);
  s->erow64.ensure(sizeof(double) * (nc + 1));
  s->t64.ensure(sizeof(double) * size_t(nc) * fd.Dpad + 64);
  launch_fill_f64(s->erow64.as<double>(), nc, 0., st);
  int64_t row0 = 0;
  for (int sI = 0; sI < fd.S; ++sI) {
    const int64_t rows = s->species_count[sI];
    const GapSpecies & g = m->segs[sI];
    if (rows > 0 && g.M > 0) {
      const double * Xs = s->X64.as<double>() + size_t(row0) * fd.Dpad;
      const double * Ts = m->T64.as<double>() + size_t(g.m0) * fd.Dpad;
      double * Kb = s->K64.as<double>();
      gemm_nt_fp64(rows, g.M, fd.D, Xs, fd.Dpad, Ts, fd.Dpad, Kb, g.M, st);
      launch_gap_pointwise_fp64(rows, g.M, Kb, g.M, m->alpha64.as<double>() + g.m0, m->zeta, Kb, g.M,
                                s->erow64.as<double>() + row0, st);
      if (forces)
        gemm_nn_fp64(rows, fd.D, g.M, Kb, g.M, Ts, fd.Dpad, s->t64.as<double>() + size_t(row0) * fd.Dpad,
                     fd.Dpad, st);
    } else if (forces && rows > 0) {
      launch_fill_f64(s->t64.as<double>() + size_t(row0) * fd.Dpad, rows * fd.Dpad, 0., st);
    }
    row0 += rows;
  }
  // struct of each sorted row
  launch_energy_reduce(nc, 0, nullptr, 0, s->erow64.as<double>(), 0, s->center_of_row.as<int32_t>(),
                       s->nl.center_struct, E_d, st);
  mark(s, 5);
  mark(s, 6);
  if (!forces) return;
  // gradients, chunked by a memory budget: materialised d c/d r and d x/d r
  const size_t per_pair = sizeof(double) * (3 * size_t(fd.D) + 3 * size_t(fd.nK));
  const size_t per_center = sizeof(double) * size_t(fd.S) * 3 * fd.nK;
  const size_t budget = plain_budget_bytes();
  ExpansionArgs ea = exp_args(c, s);
  PsArgs pa;
  pa.fd = fd;
  pa.n_centers = nc;
  pa.normalize = c->hy.normalize;
  pa.row_of_center = s->row_of_center.as<int32_t>();
  const std::vector<int64_t> & poff = pair_offsets_host(s);
  int64_t c0 = 0;
  while (c0 < nc) {
    int64_t c1 = c0;
    size_t bytes = 0;
    while (c1 < nc) {
      size_t add = per_pair * size_t(poff[c1 + 1] - poff[c1]) + per_center;
      if (c1 > c0 && bytes + add > budget) break;
      bytes += add;
      ++c1;
    }
    const int64_t p_base = poff[c0];
    const int64_t np = poff[c1] - p_base;
    s->dCp.ensure(sizeof(double) * size_t(np) * 3 * fd.nK + 64);
    s->dCs.ensure(per_center * size_t(c1 - c0) + 64);
    s->dXp.ensure(sizeof(double) * size_t(np) * 3 * fd.D + 64);
    launch_expansion_grad_fp64(ea, c0, c1, p_base, s->dCp.as<double>(), st);
    launch_expansion_selfgrad_fp64(ea, c0, c1, p_base, s->dCp.as<double>(), s->dCs.as<double>(), st);
    launch_ps_grad_fp64(pa, ea, c0, c1, p_base, s->C64.as<double>(), s->X64.as<double>(),
                        s->invn64.as<double>(), s->dCp.as<double>(), s->dCs.as<double>(),
                        s->dXp.as<double>(), st);
    launch_force_contract_fp64(fd, c0, c1, p_base, s->nl.pair_off, s->nl.pair_j,
                               s->row_of_center.as<int32_t>(), s->dXp.as<double>(), s->t64.as<double>(),
                               fd.Dpad, grad_d, st, s->nl.pair_dist, s->nl.pair_dir, s->nl.center_struct,
                               stress_d);
    c0 = c1;
  }
  mark(s, 7);
}

// Offset of species sI's energy partials ([ceil(M/256)][rows]) in epart: the
// grouped forward GEMM writes every species' partials in one launch.
int64_t eofs_of(const rgpu_structures * s, const rgpu_gap_model * m, int sI) {
  int64_t o = 0;
  for (int k = 0; k < sI; ++k) o += s->species_count[k] * ((m->segs[k].M + kTcTileN - 1) / kTcTileN);
  return o;
}

// W offsets of the species segments (rows x Mpad BF16 each) in s->Wh/Wl.
std::vector<int64_t> w_offsets(const rgpu_gap_model * m, const rgpu_structures * s) {
  std::vector<int64_t> wofs(s->fd.S);
  int64_t woff = 0;
  for (int sI = 0; sI < s->fd.S; ++sI) {
    wofs[sI] = woff;
    woff += s->species_count[sI] * m->segs[sI].Mpad;
  }
  return wofs;
}

// Rows and 128-row tiles of each central species (rows in species order).
TileMaskArgs tile_mask_args(const rgpu_structures * s) {
  TileMaskArgs a{};
  a.S = s->fd.S;
  int64_t r = 0, t = 0;
  for (int sI = 0; sI < s->fd.S; ++sI) {
    a.row0[sI] = r;
    a.rows[sI] = s->species_count[sI];
    a.tile_off[sI] = t;
    r += s->species_count[sI];
    t += (s->species_count[sI] + 127) / 128;
  }
  a.tile_off[s->fd.S] = t;
  return a;
}

// Species skipping of a grouped GEMM over the packed columns (mode 1: K, the
// forward; 2: N, the backward), for layouts of more than one species group.
void set_segments(Bf16x3Gemm & a, const rgpu_structures * s, const TileMaskArgs & tm, int sI, int mode) {
  const FeatureDims & fd = s->fd;
  if (fd.G < 2) return;
  a.seg_mode = mode;
  a.seg_G = fd.G;
  a.seg_LD = fd.lenD / 32;
  a.seg_LO = fd.lenO / 32;
  a.tile_mask = s->tile_mask.as<uint32_t>() + tm.tile_off[sI];
}

// Fast path, forward half: the grouped tcgen05 GEMM with the GAP epilogue
// (energy partials and W = alpha zeta k^(zeta-1) as a BF16 pair), then the
// per-structure energies (baseline not included).
void gap_fast_forward(rgpu_gap_model * m, rgpu_structures * s, double * E_d) {
  const FeatureDims & fd = s->fd;
  const int64_t nc = s->nl.n_centers;
  cudaStream_t st = s->st;
  s->fwd_model = nullptr;
  mark(s, 4);
  // per-species W (BF16 hi/lo) and energy partial buffers
  int64_t wtot = 0, eparts = 0;
  for (int sI = 0; sI < fd.S; ++sI) {
    wtot += s->species_count[sI] * m->segs[sI].Mpad;
    eparts += s->species_count[sI] * ((m->segs[sI].M + kTcTileN - 1) / kTcTileN);
  }
  s->Wh.ensure(sizeof(uint16_t) * size_t(std::max<int64_t>(wtot, 1)) + 64);
  s->Wl.ensure(sizeof(uint16_t) * size_t(std::max<int64_t>(wtot, 1)) + 64);
  s->epart.ensure(sizeof(float) * size_t(std::max<int64_t>(eparts, 1)) + 64);
  s->dX32.ensure(sizeof(float) * size_t(nc) * fd.Dg + 64);
  // species present in each 128-row tile (rows sorted by species and mask)
  const TileMaskArgs tm = tile_mask_args(s);
  if (fd.G > 1) {
    s->tile_mask.ensure(sizeof(uint32_t) * size_t(std::max<int64_t>(tm.tile_off[fd.S], 1)) + 64);
    launch_tile_masks(tm, s->center_of_row.as<int32_t>(), s->present.as<uint32_t>(), s->tile_mask.as<uint32_t>(), st);
  }
  const __nv_bfloat16 * Xh = s->Xh.as<__nv_bfloat16>();
  const __nv_bfloat16 * Xl = s->Xl.as<__nv_bfloat16>();
  __nv_bfloat16 * Wh = s->Wh.as<__nv_bfloat16>();
  __nv_bfloat16 * Wl = s->Wl.as<__nv_bfloat16>();
  const std::vector<int64_t> wofs = w_offsets(m, s);
  int64_t row0 = 0;
  std::vector<Bf16x3Gemm> fwd;
  for (int sI = 0; sI < fd.S; ++sI) {
    const int64_t rows = s->species_count[sI];
    const GapSpecies & g = m->segs[sI];
    if (rows > 0 && g.M > 0) {
      Bf16x3Gemm a{};
      a.M = rows;
      a.N = g.M;
      a.K = fd.Dg;
      a.A_hi = Xh + size_t(row0) * fd.Dg;
      a.A_lo = Xl + size_t(row0) * fd.Dg;
      a.lda = fd.Dg;
      a.B_hi = m->Th.as<__nv_bfloat16>() + size_t(g.m0) * fd.Dg;
      a.B_lo = m->Tl.as<__nv_bfloat16>() + size_t(g.m0) * fd.Dg;
      a.ldb = fd.Dg;
      a.epilogue = 1;
      a.W_hi = Wh + wofs[sI];
      a.W_lo = Wl + wofs[sI];
      a.ldw = g.Mpad;
      a.alpha = m->alpha32.as<float>() + g.m0;
      a.zeta = m->zeta;
      a.e_part = s->epart.as<float>() + eofs_of(s, m, sI);
      a.row_scale = s->xscale32.as<float>() + row0;  // k = (p . t) / |p|
      set_segments(a, s, tm, sI, 1);  // K blocks of species pairs absent from a tile are skipped
      fwd.push_back(a);
    }
    row0 += rows;
  }
  gemm_bf16x3_grouped(fwd.data(), int(fwd.size()), st, tile_config(fd.S, fd.n, fd.L).gemm_variant);
  row0 = 0;
  for (int sI = 0; sI < fd.S; ++sI) {
    const int64_t rows = s->species_count[sI];
    const GapSpecies & g = m->segs[sI];
    if (rows > 0 && g.M > 0) {
      const int nparts = (g.M + kTcTileN - 1) / kTcTileN;
      launch_energy_reduce(rows, nparts, s->epart.as<float>() + eofs_of(s, m, sI), rows, nullptr, row0,
                           s->center_of_row.as<int32_t>(), s->nl.center_struct, E_d, st);
    }
    row0 += rows;
  }
  mark(s, 5);
}

// Fast path, backward half: dE/dx = W T (grouped GEMM), the power-spectrum
// backward to dE/dc, then the pair adjoint into F_d (= -dE/dr) and the
// optional stress sums. With struct_scale, the contributions of every
// structure are multiplied by struct_scale[structure] (an upstream gradient
// per structure energy).
void gap_fast_backward(rgpu_gap_model * m, rgpu_structures * s, double * F_d, double * stress_d,
                       const double * struct_scale = nullptr) {
  rgpu_calculator * c = m->calc;
  const FeatureDims & fd = s->fd;
  const int64_t nc = s->nl.n_centers;
  cudaStream_t st = s->st;
  const __nv_bfloat16 * Xh = s->Xh.as<__nv_bfloat16>();
  const __nv_bfloat16 * Xl = s->Xl.as<__nv_bfloat16>();
  __nv_bfloat16 * Wh = s->Wh.as<__nv_bfloat16>();
  __nv_bfloat16 * Wl = s->Wl.as<__nv_bfloat16>();
  const std::vector<int64_t> wofs = w_offsets(m, s);
  int64_t row0 = 0;
  std::vector<Bf16x3Gemm> bwd;
  for (int sI = 0; sI < fd.S; ++sI) {
    const int64_t rows = s->species_count[sI];
    const GapSpecies & g = m->segs[sI];
    if (rows > 0 && g.M > 0) {
      Bf16x3Gemm a{};
      a.M = rows;
      a.N = fd.Dg;
      a.K = g.Mpad;
      a.A_hi = Wh + wofs[sI];
      a.A_lo = Wl + wofs[sI];
      a.lda = g.Mpad;
      a.B_hi = m->Tth.as<__nv_bfloat16>() + m->tt_off[sI];
      a.B_lo = m->Ttl.as<__nv_bfloat16>() + m->tt_off[sI];
      a.ldb = g.Mpad;
      a.epilogue = 0;
      a.C = s->dX32.as<float>() + size_t(row0) * fd.Dg;
      a.ldc = fd.Dg;
      // N tiles of species pairs absent from a tile are not computed; the
      // power-spectrum backward reads zeros for them (chunk map)
      set_segments(a, s, tile_mask_args(s), sI, 2);
      bwd.push_back(a);
    } else if (rows > 0) {
      launch_fill_f32(s->dX32.as<float>() + size_t(row0) * fd.Dg, rows * fd.Dg, 0.f, st);
    }
    row0 += rows;
  }
  gemm_bf16x3_grouped(bwd.data(), int(bwd.size()), st, tile_config(fd.S, fd.n, fd.L).gemm_variant);
  mark(s, 6);
  PsArgs pa;
  pa.fd = fd;
  pa.n_centers = nc;
  pa.normalize = c->hy.normalize;
  pa.row_of_center = s->row_of_center.as<int32_t>();
  s->dC32.ensure(sizeof(float) * size_t(nc) * fd.S * fd.nK + 64);
  s->chunk_map.ensure(sizeof(uint32_t) * size_t(fd.Dg / 4) + 64);
  launch_ps_bwd_fp32(pa, s->C32.as<float>(), Xh, Xl, s->xscale32.as<float>(), s->dX32.as<float>(),
                     s->chunk_map.as<uint32_t>(), s->present.as<uint32_t>(), s->dC32.as<float>(), st);
  if (struct_scale)
    launch_scale_rows_by_group(s->dC32.as<float>(), nc, int64_t(fd.S) * fd.nK, s->nl.center_struct, struct_scale,
                               st);
  mark(s, 7);
  ExpansionArgs ea = exp_args(c, s);
  launch_pair_adjoint_fp32(ea, s->nl.pair_center, s->nl.n_pairs, s->dC32.as<float>(), F_d, st,
                           s->nl.center_struct, stress_d);
}

void gap_fast(rgpu_gap_model * m, rgpu_structures * s, double * E_d, double * F_d, bool forces,
              double * stress_d) {
  gap_fast_forward(m, s, E_d);
  if (forces) gap_fast_backward(m, s, F_d, stress_d);
}

}  // namespace

// Cell volume as the reference computes it, from the lattice vector lengths
// and the cosines of the angles between them
// (structure_managers/atomic_structure.hh:137-155); rows of `cell` are the
// lattice vectors.
static double cell_volume(const double * cell) {
  double len[3], v[3][3];
  for (int i = 0; i < 3; ++i) {
    for (int k = 0; k < 3; ++k) v[i][k] = cell[3 * i + k];
    len[i] = std::sqrt(v[i][0] * v[i][0] + v[i][1] * v[i][1] + v[i][2] * v[i][2]);
  }
  auto dot = [&](int a, int b) { return v[a][0] * v[b][0] + v[a][1] * v[b][1] + v[a][2] * v[b][2]; };
  const double al = std::acos(dot(1, 2) / len[1] / len[2]);
  const double be = std::acos(dot(0, 2) / len[0] / len[2]);
  const double ga = std::acos(dot(1, 0) / len[1] / len[0]);
  const double c0 = std::cos(al), c1 = std::cos(be), c2 = std::cos(ga);
  return len[0] * len[1] * len[2] * std::sqrt(1 - c0 * c0 - c1 * c1 - c2 * c2 + 2 * c0 * c1 * c2);
}

extern "C" {
static void calculator_to_device(rgpu_calculator * c);
}

// Energy baseline of each structure (models/krr.py:68-90), FP64 on the host:
// a table over the atom types (validated to [0, 130) by rgpu_structures_set).
static std::vector<double> structure_baselines(const rgpu_gap_model * m, const rgpu_structures * s) {
  double sc[130] = {0.};
  for (size_t i = 0; i < m->species.size(); ++i)
    if (m->species[i] >= 0 && m->species[i] < 130) sc[m->species[i]] = m->self_contrib[i];
  std::vector<double> y0(s->n_struct, 0.);
  for (int k = 0; k < s->n_struct; ++k)
    for (int64_t a = s->atom_off[k]; a < s->atom_off[k + 1]; ++a) y0[k] += sc[s->types[a]];
  return y0;
}

// Energies, forces and (optionally) the negative stress of a GAP model: the
// reference's KRR.predict / predict_forces / predict_stress
// (bindings/rascal/models/krr.py:92-210) on the GPU.
static void gap_predict_impl(rgpu_gap_model * m, rgpu_structures * s, int precision, double * energies,
                             double * forces, double * neg_stress) {
  {
    if (!m || !s) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    if (s->has_mask)
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "Can't compute spherical expansion gradients with masked center atoms",
                  RGPU_EXC_LOGIC_ERROR);
    calculator_to_device(m->calc);
    s->timed = true;
    mark(s, 0);
    const bool want_forces = true;
    // neighbour list, layout, features
    build_nl(s, m->calc->hy.cutoff);
    mark(s, 1);
    compute_features(m->calc, s, precision, want_forces, m->species, /*need_x32=*/false);
    model_layout(m, s, precision == RGPU_PRECISION_FP32);
    const int64_t na = s->n_atoms;
    s->E_d.ensure(sizeof(double) * (s->n_struct + 1));
    s->F_d.ensure(sizeof(double) * 3 * (na + 1));
    RGPU_CUDA(cudaMemsetAsync(s->E_d.p, 0, sizeof(double) * s->n_struct, s->st));
    RGPU_CUDA(cudaMemsetAsync(s->F_d.p, 0, sizeof(double) * 3 * na, s->st));
    double * stress_d = nullptr;
    if (neg_stress) {
      s->S_d.ensure(sizeof(double) * 6 * (s->n_struct + 1));
      RGPU_CUDA(cudaMemsetAsync(s->S_d.p, 0, sizeof(double) * 6 * s->n_struct, s->st));
      stress_d = s->S_d.as<double>();
    }
    if (precision == RGPU_PRECISION_FP64)
      gap_plain(m, s, s->E_d.as<double>(), s->F_d.as<double>(), want_forces, stress_d);
    else
      gap_fast(m, s, s->E_d.as<double>(), s->F_d.as<double>(), want_forces, stress_d);
    mark(s, 8);
    // outputs through the pinned staging buffer: a device-to-host copy into
    // the caller's pageable memory is staged by the driver at a fraction of
    // the bandwidth
    const size_t eb = energies ? sizeof(double) * s->n_struct : 0, fb = forces ? sizeof(double) * 3 * na : 0,
                 sb = neg_stress ? sizeof(double) * 6 * s->n_struct : 0;
    const size_t need = eb + fb + sb + 64;
    if (need > s->pinned_cap) RGPU_CUDA(cudaStreamSynchronize(s->st));  // no copy may use the old buffer
    unsigned char * pin = static_cast<unsigned char *>(staging(s, need));
    if (eb) RGPU_CUDA(cudaMemcpyAsync(pin, s->E_d.p, eb, cudaMemcpyDeviceToHost, s->st));
    if (fb) RGPU_CUDA(cudaMemcpyAsync(pin + eb, s->F_d.p, fb, cudaMemcpyDeviceToHost, s->st));
    if (sb) RGPU_CUDA(cudaMemcpyAsync(pin + eb + fb, s->S_d.p, sb, cudaMemcpyDeviceToHost, s->st));
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    if (eb) std::memcpy(energies, pin, eb);
    if (fb) std::memcpy(forces, pin + eb, fb);
    if (sb) std::memcpy(neg_stress, pin + eb + fb, sb);
    if (precision == RGPU_PRECISION_FP32) {
      const int where = gemm_tc_timeout(true);
      if (where)
        throw Error(RGPU_ERR_TIMEOUT, "tensor-core GEMM: a bounded pipeline wait gave up (stage " +
                                          std::to_string(where) + ")");
    }
    if (energies) {
      const std::vector<double> y0 = structure_baselines(m, s);
      for (int st = 0; st < s->n_struct; ++st) energies[st] += y0[st];
    }
    if (forces && precision == RGPU_PRECISION_FP64)
      for (int64_t i = 0; i < 3 * na; ++i) forces[i] = -forces[i];
    if (neg_stress)
      for (int st = 0; st < s->n_struct; ++st) {
        const double v = cell_volume(&s->cells_h[9 * size_t(st)]);
        for (int k = 0; k < 6; ++k) neg_stress[6 * st + k] /= v;
      }
  }
}

// Forward half of the adjoint path for automatic differentiation: energies
// of the FP32 path into device memory, with everything the backward needs
// (neighbour list, features, W) left on the device. The reference computes
// energies and forces in separate calls, KRR.predict and
// KRR.predict_forces (bindings/rascal/models/krr.py:92-166).
static void gap_forward_dev_impl(rgpu_gap_model * m, rgpu_structures * s, const double * positions_dev,
                                 double * energies_dev) {
  if (!m || !s || !energies_dev) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (s->has_mask)
    throw Error(RGPU_ERR_INVALID_ARGUMENT, "Can't compute spherical expansion gradients with masked center atoms",
                RGPU_EXC_LOGIC_ERROR);
  calculator_to_device(m->calc);
  s->timed = false;
  if (positions_dev) {
    RGPU_CUDA(cudaMemcpyAsync(s->pos_d.p, positions_dev, sizeof(double) * 3 * s->n_atoms,
                              cudaMemcpyDeviceToDevice, s->st));
    s->nl_valid = false;
    s->feat_valid = false;
  }
  build_nl(s, m->calc->hy.cutoff);
  compute_features(m->calc, s, RGPU_PRECISION_FP32, true, m->species, /*need_x32=*/false);
  model_layout(m, s, true);
  s->E_d.ensure(sizeof(double) * (s->n_struct + 1));
  RGPU_CUDA(cudaMemsetAsync(s->E_d.p, 0, sizeof(double) * s->n_struct, s->st));
  gap_fast_forward(m, s, s->E_d.as<double>());
  const std::vector<double> y0 = structure_baselines(m, s);
  upload(s, s->y0_d, y0.data(), sizeof(double) * y0.size());
  launch_add_f64(s->E_d.as<double>(), s->y0_d.as<double>(), energies_dev, s->n_struct, s->st);
  RGPU_CUDA(cudaStreamSynchronize(s->st));
  const int where = gemm_tc_timeout(true);
  if (where)
    throw Error(RGPU_ERR_TIMEOUT, "tensor-core GEMM: a bounded pipeline wait gave up (stage " +
                                      std::to_string(where) + ")");
  s->fwd_model = m;
}

// Backward half: grad_dev[a][c] = sum_A energies_grad_dev[A] dE_A/dr_a[c]
// from the state the forward left: dE/dx = W T, the power-spectrum
// backward, the per-structure scaling, the pair adjoint.
static void gap_backward_dev_impl(rgpu_gap_model * m, rgpu_structures * s, const double * energies_grad_dev,
                                  double * grad_dev) {
  if (!m || !s || !energies_grad_dev || !grad_dev) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (s->fwd_model != m || !s->feat_valid || !s->nl_valid)
    throw Error(RGPU_ERR_NOT_COMPUTED, "the backward needs the forward of the same model and structures, with "
                                       "no other call on the structures in between");
  s->timed = false;
  const int64_t na = s->n_atoms;
  s->F_d.ensure(sizeof(double) * 3 * (na + 1));
  RGPU_CUDA(cudaMemsetAsync(s->F_d.p, 0, sizeof(double) * 3 * na, s->st));
  gap_fast_backward(m, s, s->F_d.as<double>(), nullptr, energies_grad_dev);
  // the adjoint accumulates forces, -dE/dr
  launch_scale_f64(s->F_d.as<double>(), -1.0, grad_dev, 3 * na, s->st);
  RGPU_CUDA(cudaStreamSynchronize(s->st));
  const int where = gemm_tc_timeout(true);
  if (where)
    throw Error(RGPU_ERR_TIMEOUT, "tensor-core GEMM: a bounded pipeline wait gave up (stage " +
                                      std::to_string(where) + ")");
}

// ---------------------------------------------------------------- training
// Sparse kernel matrices of a GAP model (models/sparse_kernels.hh), FP64.
// Their columns follow the order in which the sparse points were given.
static void kernel_features(rgpu_gap_model * m, rgpu_structures * s, bool grads) {
  if (!m || !s) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (grads && s->has_mask)
    throw Error(RGPU_ERR_INVALID_ARGUMENT, "Can't compute spherical expansion gradients with masked center atoms",
                RGPU_EXC_LOGIC_ERROR);
  calculator_to_device(m->calc);
  s->timed = false;
  build_nl(s, m->calc->hy.cutoff);
  compute_features(m->calc, s, RGPU_PRECISION_FP64, grads, m->species, /*need_x32=*/false);
  model_layout(m, s, false);
}

// K = X_s T_s^T of species sI into s->K64 (rows x M).
static void species_dots(rgpu_gap_model * m, rgpu_structures * s, int sI, int64_t row0) {
  const FeatureDims & fd = s->fd;
  const GapSpecies & g = m->segs[sI];
  const int64_t rows = s->species_count[sI];
  s->K64.ensure(sizeof(double) * size_t(std::max<int64_t>(rows, 1)) * std::max(g.M, 1) + 64);
  gemm_nt_fp64(rows, g.M, fd.D, s->X64.as<double>() + size_t(row0) * fd.Dpad, fd.Dpad,
               m->T64.as<double>() + size_t(g.m0) * fd.Dpad, fd.Dpad, s->K64.as<double>(), g.M, s->st);
}

// K_NM energy rows: SparseKernelImpl<GAP>::compute for target Structure
// (models/sparse_kernels.hh:104-131) or Atom (:165-191).
static void sparse_kernel_impl(rgpu_gap_model * m, rgpu_structures * s, bool atom_target, double * out) {
  kernel_features(m, s, false);
  const FeatureDims & fd = s->fd;
  const int64_t rows_out = atom_target ? s->nl.n_centers : s->n_struct;
  const size_t bytes = sizeof(double) * size_t(rows_out) * m->M;
  s->knm.ensure(bytes + 64);
  RGPU_CUDA(cudaMemsetAsync(s->knm.p, 0, bytes, s->st));
  int64_t row0 = 0;
  for (int sI = 0; sI < fd.S; ++sI) {
    const int64_t rows = s->species_count[sI];
    const GapSpecies & g = m->segs[sI];
    if (rows > 0 && g.M > 0) {
      species_dots(m, s, sI, row0);
      launch_knm_rows(rows, g.M, s->K64.as<double>(), m->zeta, s->center_of_row.as<int32_t>(), row0,
                      s->nl.center_struct, atom_target, m->ucol.as<int32_t>() + g.m0, s->knm.as<double>(), m->M,
                      s->st);
    }
    row0 += rows;
  }
  if (bytes) RGPU_CUDA(cudaMemcpyAsync(out, s->knm.p, bytes, cudaMemcpyDeviceToHost, s->st));
  RGPU_CUDA(cudaStreamSynchronize(s->st));
}

// K_NM gradient rows: SparseKernelImpl<GAP>::compute_derivative
// (models/sparse_kernels.hh:258-499). dX/dr is materialised chunk by chunk
// as in the plain prediction path and contracted with the sparse points of
// each central species by one gathered GEMM per species and chunk.
static void sparse_kernel_derivative_impl(rgpu_gap_model * m, rgpu_structures * s, bool neg_stress,
                                          double * out) {
  kernel_features(m, s, true);
  s->timed = true;
  for (int k = 0; k < 4; ++k) mark(s, k);
  rgpu_calculator * c = m->calc;
  const FeatureDims & fd = s->fd;
  const int64_t nc = s->nl.n_centers;
  const int M = m->M;
  cudaStream_t st = s->st;
  const int64_t rows_out = 3 * nc + (neg_stress ? 6 * int64_t(s->n_struct) : 0);
  const size_t bytes = sizeof(double) * size_t(rows_out) * M;
  s->knm.ensure(bytes + 64);
  RGPU_CUDA(cudaMemsetAsync(s->knm.p, 0, bytes, st));
  if (M == 0 || nc == 0) {
    RGPU_CUDA(cudaStreamSynchronize(st));
    return;
  }
  // zeta (X_i . T_m)^(zeta-1) of every row, species by species
  std::vector<int64_t> woff(fd.S + 1, 0), srow0(fd.S + 1, 0);
  for (int sI = 0; sI < fd.S; ++sI) {
    woff[sI + 1] = woff[sI] + s->species_count[sI] * m->segs[sI].M;
    srow0[sI + 1] = srow0[sI] + s->species_count[sI];
  }
  s->W64.ensure(sizeof(double) * size_t(std::max<int64_t>(woff[fd.S], 1)) + 64);
  mark(s, 4);
  for (int sI = 0; sI < fd.S; ++sI) {
    const int64_t rows = s->species_count[sI];
    const GapSpecies & g = m->segs[sI];
    if (rows == 0 || g.M == 0) continue;
    gemm_nt_fp64(rows, g.M, fd.D, s->X64.as<double>() + size_t(srow0[sI]) * fd.Dpad, fd.Dpad,
                 m->T64.as<double>() + size_t(g.m0) * fd.Dpad, fd.Dpad, s->W64.as<double>() + woff[sI], g.M, st);
    launch_kernel_weight(rows * g.M, s->W64.as<double>() + woff[sI], m->zeta, st);
  }
  mark(s, 5);
  mark(s, 6);
  // The reference returns from its loop over structures at the first one
  // whose centre species have no sparse points (models/sparse_kernels.hh:
  // 347-349): that structure and all later ones keep zero rows.
  std::vector<int> sp_index(130, -1);
  for (int sI = 0; sI < fd.S; ++sI) sp_index[s->species[sI]] = sI;
  int64_t c_stop = nc;
  for (int st_i = 0; st_i < s->n_struct; ++st_i) {
    bool shared = false;
    for (int64_t a = s->atom_off[st_i]; a < s->atom_off[st_i + 1] && !shared; ++a)
      shared = m->segs[sp_index[s->types[a]]].M > 0;
    if (!shared) {
      c_stop = s->atom_off[st_i];  // centres are the atoms (no centre mask with gradients)
      break;
    }
  }
  const std::vector<int64_t> & poff = pair_offsets_host(s);
  const size_t per_pair = sizeof(double) * (3 * size_t(fd.D) + 3 * size_t(fd.nK));
  const size_t per_center =
      sizeof(double) * (size_t(fd.S) * 3 * fd.nK + (neg_stress ? 6 * size_t(fd.D) : 0));
  const size_t budget = plain_budget_bytes();
  ExpansionArgs ea = exp_args(c, s);
  PsArgs pa;
  pa.fd = fd;
  pa.n_centers = nc;
  pa.normalize = c->hy.normalize;
  pa.row_of_center = s->row_of_center.as<int32_t>();
  std::vector<std::vector<int32_t>> lists(fd.S), centres(fd.S);
  int64_t c0 = 0;
  while (c0 < c_stop) {
    int64_t c1 = c0;
    size_t used = 0;
    while (c1 < c_stop) {
      size_t add = per_pair * size_t(poff[c1 + 1] - poff[c1]) + per_center;
      if (c1 > c0 && used + add > budget) break;
      used += add;
      ++c1;
    }
    const int64_t p_base = poff[c0];
    const int64_t np = poff[c1] - p_base;
    // pairs of the chunk listed by the species of their centre: (pair - p_base, centre)
    for (auto & l : lists) l.clear();
    for (auto & l : centres) l.clear();
    for (int64_t ci = c0; ci < c1; ++ci) {
      const int sI = sp_index[s->types[ci]];
      std::vector<int32_t> & l = lists[sI];
      centres[sI].push_back(int32_t(ci));
      for (int64_t p = poff[ci]; p < poff[ci + 1]; ++p) {
        l.push_back(int32_t(p - p_base));
        l.push_back(int32_t(ci));
      }
    }
    // one upload: [pair lists of all species][centre lists of all species]
    std::vector<int32_t> flat;
    std::vector<int64_t> loff(fd.S + 1, 0), coff(fd.S + 1, 0);
    for (int sI = 0; sI < fd.S; ++sI) {
      loff[sI] = int64_t(flat.size()) / 2;
      flat.insert(flat.end(), lists[sI].begin(), lists[sI].end());
    }
    loff[fd.S] = int64_t(flat.size()) / 2;
    const int64_t cbase = int64_t(flat.size());
    for (int sI = 0; sI < fd.S; ++sI) {
      coff[sI] = int64_t(flat.size()) - cbase;
      flat.insert(flat.end(), centres[sI].begin(), centres[sI].end());
    }
    coff[fd.S] = int64_t(flat.size()) - cbase;
    upload(s, s->plist, flat.data(), sizeof(int32_t) * flat.size());
    if (neg_stress) s->Vvir.ensure(sizeof(double) * 6 * size_t(fd.D) * size_t(c1 - c0) + 64);
    s->dCp.ensure(sizeof(double) * size_t(np) * 3 * fd.nK + 64);
    s->dCs.ensure(per_center * size_t(c1 - c0) + 64);
    s->dXp.ensure(sizeof(double) * size_t(np) * 3 * fd.D + 64);
    launch_expansion_grad_fp64(ea, c0, c1, p_base, s->dCp.as<double>(), st);
    launch_expansion_selfgrad_fp64(ea, c0, c1, p_base, s->dCp.as<double>(), s->dCs.as<double>(), st);
    launch_ps_grad_fp64(pa, ea, c0, c1, p_base, s->C64.as<double>(), s->X64.as<double>(), s->invn64.as<double>(),
                        s->dCp.as<double>(), s->dCs.as<double>(), s->dXp.as<double>(), st);
    for (int sI = 0; sI < fd.S; ++sI) {
      const GapSpecies & g = m->segs[sI];
      const int64_t n_list = loff[sI + 1] - loff[sI];
      if (n_list == 0 || g.M == 0) continue;
      KnmDerArgs a{};
      a.list = s->plist.as<int32_t>() + 2 * loff[sI];
      a.n_list = n_list;
      a.p_base = p_base;
      a.dX = s->dXp.as<double>();
      a.D = fd.D;
      a.T = m->T64.as<double>() + size_t(g.m0) * fd.Dpad;
      a.ldt = fd.Dpad;
      a.M = g.M;
      a.W = s->W64.as<double>() + woff[sI];
      a.row0 = srow0[sI];
      a.row_of_center = s->row_of_center.as<int32_t>();
      a.pair_j = s->nl.pair_j;
      a.ucol = m->ucol.as<int32_t>() + g.m0;
      a.out = s->knm.as<double>();
      a.ldo = M;
      launch_knm_derivative(a, st);
      if (neg_stress) {
        KnmStressArgs b{};
        b.centres = s->plist.as<int32_t>() + cbase + coff[sI];
        b.n_centres = coff[sI + 1] - coff[sI];
        b.p_base = p_base;
        b.pair_off = s->nl.pair_off;
        b.pair_dist = s->nl.pair_dist;
        b.pair_dir = s->nl.pair_dir;
        b.dX = s->dXp.as<double>();
        b.D = fd.D;
        b.V = s->Vvir.as<double>();
        b.T = a.T;
        b.ldt = a.ldt;
        b.M = g.M;
        b.W = a.W;
        b.row0 = a.row0;
        b.row_of_center = a.row_of_center;
        b.center_struct = s->nl.center_struct;
        b.ucol = a.ucol;
        b.out = a.out;
        b.ldo = M;
        b.stress_row0 = 3 * nc;
        launch_knm_stress(b, st);
      }
    }
    c0 = c1;
  }
  mark(s, 7);
  mark(s, 8);
  RGPU_CUDA(cudaMemcpyAsync(out, s->knm.p, bytes, cudaMemcpyDeviceToHost, st));
  RGPU_CUDA(cudaStreamSynchronize(st));
  if (neg_stress)
    for (int st_i = 0; st_i < s->n_struct; ++st_i) {
      const double v = cell_volume(&s->cells_h[9 * size_t(st_i)]);
      double * r = out + size_t(3 * nc + 6 * int64_t(st_i)) * M;
      for (int k = 0; k < 6 * M; ++k) r[k] /= v;
    }
}

// K_MM: SparseKernel::compute(sparse_points) (models/sparse_kernels.hh:
// 141-156, models/sparse_points.hh:144-170), one FP64 T_s T_s^T per species.
static void sparse_kernel_mm_impl(rgpu_gap_model * m, double * out) {
  if (!m) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
  const int M = m->M;
  if (M == 0) return;
  const int Sm = int(m->species.size());
  const FeatureDims fm = make_dims(m->calc->hy, Sm);
  std::vector<int32_t> order;
  std::vector<int> m0(Sm + 1, 0);
  for (int a = 0; a < Sm; ++a) {
    m0[a] = int(order.size());
    for (int r = 0; r < M; ++r)
      if (m->sp_species[r] == m->species[a]) order.push_back(r);
  }
  m0[Sm] = int(order.size());
  std::vector<double> T(size_t(M) * fm.D);
  for (int k = 0; k < M; ++k)
    std::memcpy(&T[size_t(k) * fm.D], &m->T[size_t(order[k]) * fm.D], sizeof(double) * fm.D);
  int Mmax = 0;
  for (int a = 0; a < Sm; ++a) Mmax = std::max(Mmax, m0[a + 1] - m0[a]);
  cudaStream_t st = nullptr;
  RGPU_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
  } guard_st{st};
  DevBuf Td, Kd, Od, Ud;
  Td.ensure(sizeof(double) * T.size());
  Kd.ensure(sizeof(double) * size_t(Mmax) * Mmax + 64);
  Od.ensure(sizeof(double) * size_t(M) * M);
  Ud.ensure(sizeof(int32_t) * order.size());
  RGPU_CUDA(cudaMemcpyAsync(Td.p, T.data(), sizeof(double) * T.size(), cudaMemcpyHostToDevice, st));
  RGPU_CUDA(cudaMemcpyAsync(Ud.p, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice, st));
  RGPU_CUDA(cudaMemsetAsync(Od.p, 0, sizeof(double) * size_t(M) * M, st));
  for (int a = 0; a < Sm; ++a) {
    const int Ms = m0[a + 1] - m0[a];
    if (Ms == 0) continue;
    const double * Ts = Td.as<double>() + size_t(m0[a]) * fm.D;
    gemm_nt_fp64(Ms, Ms, fm.D, Ts, fm.D, Ts, fm.D, Kd.as<double>(), Ms, st);
    launch_kmm_scatter(Ms, Kd.as<double>(), m->zeta, Ud.as<int32_t>() + m0[a], Od.as<double>(), M, st);
  }
  RGPU_CUDA(cudaMemcpyAsync(out, Od.p, sizeof(double) * size_t(M) * M, cudaMemcpyDeviceToHost, st));
  RGPU_CUDA(cudaStreamSynchronize(st));
}

// ------------------------------------------------------------------ MD step
// A step of a molecular-dynamics loop on a fixed set of structures: the FP32
// path from new positions to energies, forces (and the negative stress),
// with no host synchronisation inside, so that it is recorded once as a
// CUDA graph and then replayed. The neighbour list is built to capacities
// 25 % above the counts of the step that recorded the graph; when a step
// outgrows them (status 104) it is recomputed by the ordinary path and the
// graph is recorded again.
// Addresses of every device buffer a recorded step can use: those of the
// structures handle (neighbour-list work included), of the model and of its
// calculator. The recording is replayed only while none of them moved.
static std::vector<const void *> md_buffers(const rgpu_gap_model * m, const rgpu_structures * s) {
  std::vector<const void *> v;
  for (const DevBuf * b : {&s->atom_off_d, &s->pos_d, &s->types_d, &s->cells_d, &s->pbc_d, &s->tag2idx_d,
                           &s->ncent_d, &s->center_off_d, &s->atom_struct_d, &s->lut, &s->row_of_center,
                           &s->center_of_row, &s->species_count_d, &s->sort_tmp, &s->present, &s->tile_mask,
                           &s->C64, &s->X64,
                           &s->invn64, &s->C32, &s->X32, &s->xscale32, &s->E_d, &s->F_d, &s->S_d, &s->K64,
                           &s->t64, &s->erow64, &s->Wh, &s->Wl, &s->dX32, &s->dC32, &s->epart, &s->Xh, &s->Xl,
                           &s->chunk_map, &s->dCp, &s->dCs, &s->dXp, &s->knm, &s->W64, &s->plist, &s->Vvir})
    v.push_back(b->p);
  const NlWork & w = s->nlw;
  for (const DevBuf * b : {&w.geom, &w.counts64, &w.scan_tmp, &w.ghost_off, &w.site_x, &w.site_type, &w.site_real,
                           &w.site_shift, &w.site_box, &w.box_base, &w.box_count, &w.box_ptr, &w.box_fill,
                           &w.sorted, &w.sorted_x, &w.sorted_info, &w.pair_count, &w.center_atom,
                           &w.center_struct, &w.pair_off, &w.pair_j, &w.pair_shift, &w.pair_dist, &w.pair_dir,
                           &w.pair_center})
    v.push_back(b->p);
  for (const DevBuf * b : {&m->T64, &m->alpha64, &m->Th, &m->Tl, &m->Tth, &m->Ttl, &m->alpha32, &m->ucol})
    v.push_back(b->p);
  const rgpu_calculator * c = m->calc;
  for (const DevBuf * b : {&c->grid, &c->y, &c->y2h, &c->yf, &c->y2hf, &c->q4f, &c->center}) v.push_back(b->p);
  return v;
}

static void md_drop(rgpu_structures * s) {
  if (s->md_exec) cudaGraphExecDestroy(s->md_exec);
  if (s->md_graph) cudaGraphDestroy(s->md_graph);
  s->md_exec = nullptr;
  s->md_graph = nullptr;
  s->md_model = nullptr;
}

// The FP32 prediction on the structures' stream with no host
// synchronisation, so that it can be recorded: positions from pinned
// pos_h (null: those already on the device), the neighbour list to `caps`,
// outputs (energies, forces, stress sums) into pinned out_h (null: left on
// the device), and the status word copied to the host at the end.
static void graph_enqueue(rgpu_gap_model * m, rgpu_structures * s, bool stress, const double * pos_h,
                          double * out_h, const NlCaps & caps) {
  rgpu_calculator * c = m->calc;
  cudaStream_t st = s->st;
  const int64_t na = s->n_atoms;
  if (pos_h) RGPU_CUDA(cudaMemcpyAsync(s->pos_d.p, pos_h, sizeof(double) * 3 * na, cudaMemcpyHostToDevice, st));
  NlInputs in;
  in.n_struct = s->n_struct;
  in.n_atoms = na;
  in.atom_off = s->atom_off_d.as<int64_t>();
  in.pos = s->pos_d.as<double>();
  in.types = s->types_d.as<int32_t>();
  in.cells = s->cells_d.as<double>();
  in.pbc = s->pbc_d.as<int32_t>();
  in.tag2idx = nullptr;
  in.n_centers = s->ncent_d.as<int32_t>();
  in.center_off = s->center_off_d.as<int64_t>();
  in.atom_struct = s->atom_struct_d.as<int32_t>();
  in.n_centers_total = s->center_off_h[s->n_struct];
  build_neighbour_list(in, c->hy.cutoff, s->nlw, s->nl, s->status_d, s->status_h, st, &caps);
  // features (the FP32 branch of compute_features, layout unchanged)
  sort_rows(s);
  const int64_t nc = s->nl.n_centers;
  const FeatureDims & fd = s->fd;
  ExpansionArgs ea = exp_args(c, s);
  PsArgs pa;
  pa.fd = fd;
  pa.n_centers = nc;
  pa.normalize = c->hy.normalize;
  pa.row_of_center = s->row_of_center.as<int32_t>();
  launch_expansion_fp32(ea, s->C32.as<float>(), s->present.as<uint32_t>(), st);
  sort_rows_by_mask(s);
  pa.present = s->present.as<uint32_t>();
  launch_ps_fwd_fast(pa, s->C32.as<float>(), nullptr, s->Xh.as<__nv_bfloat16>(), s->Xl.as<__nv_bfloat16>(),
                     s->xscale32.as<float>(), st);
  RGPU_CUDA(cudaMemsetAsync(s->E_d.p, 0, sizeof(double) * s->n_struct, st));
  RGPU_CUDA(cudaMemsetAsync(s->F_d.p, 0, sizeof(double) * 3 * na, st));
  if (stress) RGPU_CUDA(cudaMemsetAsync(s->S_d.p, 0, sizeof(double) * 6 * s->n_struct, st));
  gap_fast(m, s, s->E_d.as<double>(), s->F_d.as<double>(), true, stress ? s->S_d.as<double>() : nullptr);
  if (double * out = out_h) {
    RGPU_CUDA(cudaMemcpyAsync(out, s->E_d.p, sizeof(double) * s->n_struct, cudaMemcpyDeviceToHost, st));
    RGPU_CUDA(cudaMemcpyAsync(out + s->n_struct, s->F_d.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost, st));
    if (stress)
      RGPU_CUDA(cudaMemcpyAsync(out + s->n_struct + 3 * na, s->S_d.p, sizeof(double) * 6 * s->n_struct,
                                cudaMemcpyDeviceToHost, st));
  }
  RGPU_CUDA(cudaMemcpyAsync(s->status_h, s->status_d, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
}

// The step's work on the structures' stream, positions from s->md_pos_h.
static void md_enqueue(rgpu_gap_model * m, rgpu_structures * s, bool stress) {
  graph_enqueue(m, s, stress, s->md_pos_h, s->md_out_h, s->md_caps);
}

// Kernel nodes of a recorded graph (the kernels one replay launches).
static int64_t graph_kernels(cudaGraph_t g) {
  size_t n = 0;
  int64_t k = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) == cudaSuccess && n > 0) {
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) == cudaSuccess)
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
      }
  }
  return k;
}

// Energy baseline and cell volume, as in gap_predict_impl.
static void md_finish(const rgpu_gap_model * m, const rgpu_structures * s, double * energies, double * forces,
                      double * neg_stress) {
  const int64_t na = s->n_atoms;
  const double * out = s->md_out_h;
  if (energies) {
    double sc[130] = {0.};
    for (size_t i = 0; i < m->species.size(); ++i)
      if (m->species[i] >= 0 && m->species[i] < 130) sc[m->species[i]] = m->self_contrib[i];
    for (int st = 0; st < s->n_struct; ++st) {
      double y0 = 0.;
      for (int64_t a = s->atom_off[st]; a < s->atom_off[st + 1]; ++a) y0 += sc[s->types[a]];
      energies[st] = out[st] + y0;
    }
  }
  if (forces) std::memcpy(forces, out + s->n_struct, sizeof(double) * 3 * na);
  if (neg_stress)
    for (int st = 0; st < s->n_struct; ++st) {
      const double v = cell_volume(&s->cells_h[9 * size_t(st)]);
      for (int k = 0; k < 6; ++k) neg_stress[6 * st + k] = out[s->n_struct + 3 * na + 6 * st + k] / v;
    }
}

static void md_step_impl(rgpu_gap_model * m, rgpu_structures * s, const double * positions, double * energies,
                         double * forces, double * neg_stress) {
  if (!m || !s || !positions) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
  const bool stress = neg_stress != nullptr;
  const int64_t na = s->n_atoms;
  ensure_stream(s);
  bool replay = false;
  if (s->md_exec) {
    if (s->md_model != m || s->md_stress != stress || m->layout_species != s->species ||
        s->md_species != s->species)
      s->md_reason = 3;
    else if (md_buffers(m, s) != s->md_buffers)
      s->md_reason = 1;
    else
      replay = true;
  }
  if (replay) {
    std::memcpy(s->md_pos_h, positions, sizeof(double) * 3 * na);
    RGPU_CUDA(cudaGraphLaunch(s->md_exec, s->st));
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    ++s->md_replays;
    const int where = gemm_tc_timeout(true);
    if (where)
      throw Error(RGPU_ERR_TIMEOUT, "tensor-core GEMM: a bounded pipeline wait gave up (stage " +
                                        std::to_string(where) + ")");
    if (s->status_h->code == 0) {
      md_finish(m, s, energies, forces, neg_stress);
      return;
    }
    // outgrown capacities or an input error: the ordinary path below
    // rebuilds, or reports the error with its message
    s->md_reason = 100 + s->status_h->code;
    RGPU_CUDA(cudaMemsetAsync(s->status_d, 0, sizeof(DevStatus), s->st));
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    s->status_h->code = 0;
  }
  md_drop(s);
  // the ordinary path: checks the input, sizes every buffer, gives this step's results
  upload(s, s->pos_d, positions, sizeof(double) * 3 * na);
  s->nl_valid = false;
  s->feat_valid = false;
  gap_predict_impl(m, s, RGPU_PRECISION_FP32, energies, forces, neg_stress);
  if (s->md_no_graph) return;
  // capacities 25 % above this step's counts
  int64_t sites = 0, boxes = 0;
  neighbour_list_counts(s->nlw, sites, boxes);
  s->md_caps.sites = sites + sites / 4 + 64;
  s->md_caps.boxes = boxes + boxes / 4 + 64;
  s->md_caps.pairs = s->nl.n_pairs + s->nl.n_pairs / 4 + 256;
  if (s->md_pos_cap < size_t(3 * na)) {
    if (s->md_pos_h) cudaFreeHost(s->md_pos_h);
    RGPU_CUDA(cudaMallocHost(&s->md_pos_h, sizeof(double) * 3 * std::max<int64_t>(na, 1)));
    s->md_pos_cap = size_t(3 * na);
  }
  const size_t nout = size_t(s->n_struct) * 7 + 3 * size_t(na);
  if (s->md_out_cap < nout) {
    if (s->md_out_h) cudaFreeHost(s->md_out_h);
    RGPU_CUDA(cudaMallocHost(&s->md_out_h, sizeof(double) * std::max<size_t>(nout, 1)));
    s->md_out_cap = nout;
  }
  if (stress) s->S_d.ensure(sizeof(double) * 6 * (s->n_struct + 1));
  std::memcpy(s->md_pos_h, positions, sizeof(double) * 3 * na);
  // one run without recording sizes the capacity buffers (no allocation may
  // happen while recording) and checks that the step fits them
  s->timed = false;
  md_enqueue(m, s, stress);
  RGPU_CUDA(cudaStreamSynchronize(s->st));
  if (s->status_h->code != 0 || gemm_tc_timeout(true)) {
    // cannot happen with fresh capacities unless something is off: leave
    // the step to the ordinary path next time
    RGPU_CUDA(cudaMemsetAsync(s->status_d, 0, sizeof(DevStatus), s->st));
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    s->status_h->code = 0;
    return;
  }
  // record; a step that cannot be recorded keeps the ordinary path
  bool ok = cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    try {
      md_enqueue(m, s, stress);
    } catch (...) {
      ok = false;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s->st, &g);
    ok = ok && e == cudaSuccess && g != nullptr;
    if (ok) {
      s->md_graph = g;
      ok = cudaGraphInstantiate(&s->md_exec, s->md_graph, 0) == cudaSuccess;
    } else if (g) {
      cudaGraphDestroy(g);
    }
  }
  if (!ok) {
    (void)cudaGetLastError();
    md_drop(s);
    s->md_no_graph = true;
    s->nl_valid = false;
    s->feat_valid = false;
    return;
  }
  s->md_model = m;
  s->md_stress = stress;
  s->md_buffers = md_buffers(m, s);
  s->md_species = s->species;
  s->md_kernels = graph_kernels(s->md_graph);
  s->md_replays = 0;
  // the ordinary step above already produced this call's results; the
  // positions of the next step arrive in md_pos_h
  s->nl_valid = false;
  s->feat_valid = false;
}

// ------------------------------------------------- predictions as CUDA graphs
static void pgraph_release(PredictGraph & g) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  if (g.out_h) cudaFreeHost(g.out_h);
  g = PredictGraph{};
}

static std::vector<int64_t> centres_per_species(const rgpu_structures * s) {
  std::vector<int64_t> c(s->species.size());
  for (size_t i = 0; i < s->species.size(); ++i) c[i] = s->centres_of_type[s->species[i]];
  return c;
}

// Outputs of a replay, from its pinned copy: baseline added to the
// energies, stress sums divided by the cell volumes (as gap_predict_impl).
static void pgraph_outputs(const rgpu_gap_model * m, const rgpu_structures * s, const PredictGraph & g,
                           double * energies, double * forces, double * neg_stress) {
  const int64_t na = s->n_atoms;
  const double * out = g.out_h;
  if (energies) {
    const std::vector<double> y0 = structure_baselines(m, s);
    for (int k = 0; k < s->n_struct; ++k) energies[k] = out[k] + y0[k];
  }
  if (forces) std::memcpy(forces, out + s->n_struct, sizeof(double) * 3 * na);
  if (neg_stress)
    for (int k = 0; k < s->n_struct; ++k) {
      const double v = cell_volume(&s->cells_h[9 * size_t(k)]);
      for (int j = 0; j < 6; ++j) neg_stress[6 * k + j] = out[s->n_struct + 3 * na + 6 * k + j] / v;
    }
}

// Replays the recorded graph of this call's size bucket, if there is one:
// true when it produced the call's results. A replay whose neighbour list
// outgrew its capacities, or whose input is invalid, drops the recording and
// leaves the call to the ordinary path (which reports input errors with the
// reference's messages).
static bool pgraph_replay(rgpu_gap_model * m, rgpu_structures * s, bool stress, double * energies,
                          double * forces, double * neg_stress) {
  if (s->pgraphs.empty()) return false;
  calculator_to_device(m->calc);
  set_layout(s, m->calc->hy, m->species);
  model_layout(m, s, true);
  const bool outputs = energies || forces || neg_stress;
  const std::vector<int64_t> cnt = centres_per_species(s);
  std::vector<const void *> bufs;
  for (PredictGraph & g : s->pgraphs) {
    if (g.model != m || g.stress != stress || g.outputs != outputs || g.n_struct != s->n_struct ||
        g.n_atoms != s->n_atoms || g.species != s->species || g.species_count != cnt)
      continue;
    if (bufs.empty()) bufs = md_buffers(m, s);
    if (g.buffers != bufs) continue;
    s->timed = false;
    RGPU_CUDA(cudaGraphLaunch(g.exec, s->st));
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    // the list on the device is the capacity-bound one: nothing computed here
    // is reused by a later call
    s->nl_valid = false;
    s->feat_valid = false;
    s->fwd_model = nullptr;
    const int where = gemm_tc_timeout(true);
    if (where)
      throw Error(RGPU_ERR_TIMEOUT, "tensor-core GEMM: a bounded pipeline wait gave up (stage " +
                                        std::to_string(where) + ")");
    if (s->status_h->code != 0) {
      RGPU_CUDA(cudaMemsetAsync(s->status_d, 0, sizeof(DevStatus), s->st));
      RGPU_CUDA(cudaStreamSynchronize(s->st));
      s->status_h->code = 0;
      pgraph_release(g);
      s->pgraphs.erase(s->pgraphs.begin() + (&g - s->pgraphs.data()));
      return false;
    }
    g.used = ++s->pgraph_clock;
    ++s->pgraph_replays;
    s->pgraph_last_kernels = g.kernels;
    pgraph_outputs(m, s, g, energies, forces, neg_stress);
    return true;
  }
  return false;
}

// Records this call's size bucket after an ordinary FP32 prediction: one run
// to the new capacities without recording (it sizes every buffer, since
// nothing may be allocated while recording, and checks that the call fits
// them), then the recording. A failure leaves the handle on the ordinary
// path for this bucket.
static void pgraph_record(rgpu_gap_model * m, rgpu_structures * s, bool stress, bool outputs) {
  constexpr size_t kMaxGraphs = 4;
  PredictGraph g;
  int64_t sites = 0, boxes = 0;
  neighbour_list_counts(s->nlw, sites, boxes);
  g.caps.sites = sites + sites / 8 + 64;
  g.caps.boxes = boxes + boxes / 8 + 64;
  g.caps.pairs = s->nl.n_pairs + s->nl.n_pairs / 8 + 256;
  g.model = m;
  g.stress = stress;
  g.outputs = outputs;
  g.n_struct = s->n_struct;
  g.n_atoms = s->n_atoms;
  g.species = s->species;
  g.species_count = centres_per_species(s);
  if (outputs) {
    const size_t nout = size_t(s->n_struct) * 7 + 3 * size_t(s->n_atoms) + 1;
    RGPU_CUDA(cudaMallocHost(&g.out_h, sizeof(double) * nout));
  }
  if (stress) s->S_d.ensure(sizeof(double) * 6 * (s->n_struct + 1));
  s->timed = false;
  bool ok = true;
  try {
    graph_enqueue(m, s, stress, nullptr, g.out_h, g.caps);
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    ok = s->status_h->code == 0 && gemm_tc_timeout(true) == 0;
  } catch (...) {
    ok = false;
  }
  if (ok) {
    ok = cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      try {
        graph_enqueue(m, s, stress, nullptr, g.out_h, g.caps);
      } catch (...) {
        ok = false;
      }
      cudaGraph_t gr = nullptr;
      const cudaError_t e = cudaStreamEndCapture(s->st, &gr);
      ok = ok && e == cudaSuccess && gr != nullptr;
      if (gr) g.graph = gr;
      ok = ok && cudaGraphInstantiate(&g.exec, g.graph, 0) == cudaSuccess;
    }
  }
  s->nl_valid = false;
  s->feat_valid = false;
  s->fwd_model = nullptr;
  if (!ok) {
    (void)cudaGetLastError();
    RGPU_CUDA(cudaMemsetAsync(s->status_d, 0, sizeof(DevStatus), s->st));
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    s->status_h->code = 0;
    pgraph_release(g);
    return;
  }
  g.buffers = md_buffers(m, s);
  g.kernels = graph_kernels(g.graph);
  g.used = ++s->pgraph_clock;
  if (s->pgraphs.size() >= kMaxGraphs) {
    auto lru = std::min_element(s->pgraphs.begin(), s->pgraphs.end(),
                                [](const PredictGraph & a, const PredictGraph & b) { return a.used < b.used; });
    pgraph_release(*lru);
    s->pgraphs.erase(lru);
  }
  s->pgraphs.push_back(g);
  ++s->pgraph_records;
}

// rgpu_gap_predict(_stress): FP32 calls go through the recorded graph of
// their size bucket when one exists, otherwise through the ordinary path,
// after which the bucket is recorded.
static void gap_predict_entry(rgpu_gap_model * m, rgpu_structures * s, int precision, double * energies,
                              double * forces, double * neg_stress) {
  if (!m || !s) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
  const bool graphs = precision == RGPU_PRECISION_FP32 && s->use_graphs && !s->has_mask;
  const bool stress = neg_stress != nullptr;
  if (graphs && pgraph_replay(m, s, stress, energies, forces, neg_stress)) return;
  gap_predict_impl(m, s, precision, energies, forces, neg_stress);
  if (graphs) pgraph_record(m, s, stress, energies || forces || neg_stress);
}

// ===================================================================== C ABI
extern "C" {

const char * rgpu_last_error(void) { return t_err.c_str(); }
int rgpu_error_kind(void) { return t_kind; }
int rgpu_version(void) { return 1; }

rgpu_status rgpu_calculator_create(const char * kind, const char * hypers_json, rgpu_calculator ** out) {
  return guard([&] {
    if (!kind || !hypers_json || !out) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    auto c = std::make_unique<rgpu_calculator>();
    parse_hypers(kind, hypers_json, c->hy);
    build_radial_spline(c->hy, c->spline);
    *out = c.release();
  });
}

rgpu_status rgpu_calculator_destroy(rgpu_calculator * calc) {
  return guard([&] { delete calc; });
}

// Device copies of the radial table, made on first use so that a calculator
// can be built (and its FP64 table inspected) on a host without a GPU.
static void calculator_to_device(rgpu_calculator * c) {
  bind_device(c->device, "the calculator");
  if (c->dev.y) return;
  {
    const RadialSpline & sp = c->spline;
    const size_t GW = size_t(sp.grid_size) * sp.width;
    std::vector<float> yf(GW), y2hf(GW);
    for (size_t i = 0; i < GW; ++i) {
      yf[i] = float(sp.y[i]);
      y2hf[i] = float(sp.y2h[i]);
    }
    // interval table of the FP32 path: one 16-byte load per channel
    const size_t W = size_t(sp.width);
    std::vector<float> q4(size_t(std::max(sp.grid_size - 1, 1)) * W * 4, 0.f);
    for (int k = 0; k + 1 < sp.grid_size; ++k)
      for (size_t c = 0; c < W; ++c) {
        float * o = &q4[(size_t(k) * W + c) * 4];
        o[0] = yf[size_t(k) * W + c];
        o[1] = y2hf[size_t(k) * W + c];
        o[2] = yf[size_t(k + 1) * W + c];
        o[3] = y2hf[size_t(k + 1) * W + c];
      }
    std::vector<double> center(sp.center.size());
    for (size_t i = 0; i < center.size(); ++i) center[i] = sp.center[i] / std::sqrt(4.0 * kPi);
    auto put = [](DevBuf & b, const void * src, size_t bytes) {
      b.ensure(bytes);
      RGPU_CUDA(cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice));
    };
    put(c->grid, sp.grid.data(), sizeof(double) * sp.grid.size());
    put(c->y, sp.y.data(), sizeof(double) * GW);
    put(c->y2h, sp.y2h.data(), sizeof(double) * GW);
    put(c->yf, yf.data(), sizeof(float) * GW);
    put(c->y2hf, y2hf.data(), sizeof(float) * GW);
    put(c->q4f, q4.data(), sizeof(float) * q4.size());
    put(c->center, center.data(), sizeof(double) * center.size());
    c->dev.grid = c->grid.as<double>();
    c->dev.y = c->y.as<double>();
    c->dev.y2h = c->y2h.as<double>();
    c->dev.yf = c->yf.as<float>();
    c->dev.y2hf = c->y2hf.as<float>();
    c->dev.q4f = c->q4f.as<float4>();
    c->dev.x1 = sp.x1;
    c->dev.h = sp.h;
    c->dev.inv_h = 1.0 / sp.h;
    c->dev.ppu = sp.points_per_unit;
    c->dev.search_size = sp.search_size;
    c->dev.W = sp.width;
  }
}

rgpu_status rgpu_calculator_name(const rgpu_calculator * calc, char * buf, size_t buflen) {
  return guard([&] {
    if (!calc || !buf) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    std::snprintf(buf, buflen, "%s", calc->hy.name.c_str());
  });
}

rgpu_status rgpu_calculator_spline_shape(const rgpu_calculator * calc, int32_t * grid_size, int32_t * width) {
  return guard([&] {
    *grid_size = calc->spline.grid_size;
    *width = calc->spline.width;
  });
}

rgpu_status rgpu_calculator_spline_table(const rgpu_calculator * calc, double * grid, double * y, double * y2h) {
  return guard([&] {
    const RadialSpline & s = calc->spline;
    if (grid) std::memcpy(grid, s.grid.data(), sizeof(double) * s.grid.size());
    if (y) std::memcpy(y, s.y.data(), sizeof(double) * s.y.size());
    if (y2h) std::memcpy(y2h, s.y2h.data(), sizeof(double) * s.y2h.size());
  });
}

rgpu_status rgpu_structures_create(rgpu_structures ** out) {
  return guard([&] {
    auto s = std::make_unique<rgpu_structures>();
    ensure_stream(s.get());
    *out = s.release();
  });
}

rgpu_status rgpu_structures_destroy(rgpu_structures * s) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!s) return;
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->md_exec) cudaGraphExecDestroy(s->md_exec);
    if (s->md_graph) cudaGraphDestroy(s->md_graph);
    for (PredictGraph & g : s->pgraphs) pgraph_release(g);
    if (s->md_pos_h) cudaFreeHost(s->md_pos_h);
    if (s->md_out_h) cudaFreeHost(s->md_out_h);
    if (s->pinned) cudaFreeHost(s->pinned);
    if (s->status_h) cudaFreeHost(s->status_h);
    if (s->status_d) cudaFree(s->status_d);
    for (auto & e : s->ev)
      if (e) cudaEventDestroy(e);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
  });
}

rgpu_status rgpu_structures_set(rgpu_structures * s, int32_t n_structures, const int64_t * atom_offsets,
                                const double * positions, const int32_t * numbers, const double * cells,
                                const int32_t * pbc, const uint8_t * center_mask) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!s || n_structures < 0 || !atom_offsets) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    md_drop(s);
    s->md_no_graph = false;
    ensure_stream(s);
    s->n_struct = n_structures;
    s->atom_off.assign(atom_offsets, atom_offsets + n_structures + 1);
    if (s->atom_off[0] != 0) throw Error(RGPU_ERR_INVALID_ARGUMENT, "atom_offsets must start at 0");
    for (int i = 0; i < n_structures; ++i)
      if (s->atom_off[i + 1] < s->atom_off[i]) throw Error(RGPU_ERR_INVALID_ARGUMENT, "atom_offsets must be non-decreasing");
    s->n_atoms = s->atom_off[n_structures];
    if (s->n_atoms > (int64_t(1) << 31) - 1) throw Error(RGPU_ERR_INVALID_ARGUMENT, "too many atoms");
    s->types.assign(numbers, numbers + s->n_atoms);
    s->cells_h.assign(cells, cells + 9 * size_t(n_structures));
    bool seen[130] = {false};
    for (int64_t a = 0; a < s->n_atoms; ++a) {
      if (s->types[a] < 0 || s->types[a] >= 130)
        throw Error(RGPU_ERR_STRUCTURE, "atom types (or atomic numbers) should be in the range [0, 130].");
      seen[s->types[a]] = true;
    }
    s->batch_species.clear();
    for (int z = 0; z < 130; ++z)
      if (seen[z]) s->batch_species.push_back(z);
    s->has_mask = false;
    if (center_mask)
      for (int64_t a = 0; a < s->n_atoms; ++a)
        if (!center_mask[a]) s->has_mask = true;
    std::fill(s->centres_of_type, s->centres_of_type + 130, int64_t(0));
    for (int64_t a = 0; a < s->n_atoms; ++a)
      if (!center_mask || center_mask[a]) ++s->centres_of_type[s->types[a]];
    std::vector<int32_t> ncent(n_structures), astruct(s->n_atoms);
    s->center_off_h.assign(n_structures + 1, 0);
    std::vector<int32_t> tag2idx;
    if (s->has_mask) tag2idx.resize(s->n_atoms);
    for (int i = 0; i < n_structures; ++i) {
      int64_t a0 = s->atom_off[i], a1 = s->atom_off[i + 1];
      int nc = 0;
      for (int64_t a = a0; a < a1; ++a) {
        astruct[a] = i;
        if (!center_mask || center_mask[a]) ++nc;
      }
      ncent[i] = nc;
      s->center_off_h[i + 1] = s->center_off_h[i] + nc;
      if (s->has_mask) {
        int64_t t = a0;
        for (int64_t a = a0; a < a1; ++a)
          if (center_mask[a]) tag2idx[t++] = int32_t(a);
        for (int64_t a = a0; a < a1; ++a)
          if (!center_mask[a]) tag2idx[t++] = int32_t(a);
      }
    }
    std::vector<Upload> ups = {
        {&s->atom_off_d, s->atom_off.data(), sizeof(int64_t) * (n_structures + 1)},
        {&s->pos_d, positions, sizeof(double) * 3 * s->n_atoms},
        {&s->types_d, numbers, sizeof(int32_t) * s->n_atoms},
        {&s->cells_d, cells, sizeof(double) * 9 * n_structures},
        {&s->pbc_d, pbc, sizeof(int32_t) * 3 * n_structures},
        {&s->ncent_d, ncent.data(), sizeof(int32_t) * n_structures},
        {&s->center_off_d, s->center_off_h.data(), sizeof(int64_t) * (n_structures + 1)},
        {&s->atom_struct_d, astruct.data(), sizeof(int32_t) * s->n_atoms}};
    if (s->has_mask) ups.push_back({&s->tag2idx_d, tag2idx.data(), sizeof(int32_t) * s->n_atoms});
    upload_many(s, ups);
    s->nl_valid = false;
    s->feat_valid = false;
    s->fwd_model = nullptr;
  });
}

rgpu_status rgpu_structures_update_positions(rgpu_structures * s, const double * positions) {
  return guard([&] {
    OnDevice on_dev(s);
    upload(s, s->pos_d, positions, sizeof(double) * 3 * s->n_atoms);
    s->nl_valid = false;
    s->feat_valid = false;
    s->fwd_model = nullptr;
  });
}

rgpu_status rgpu_structures_invalidate(rgpu_structures * s) {
  return guard([&] {
    OnDevice on_dev(s);
    s->nl_valid = false;
    s->feat_valid = false;
    s->fwd_model = nullptr;
  });
}

rgpu_status rgpu_structures_stream(const rgpu_structures * s, void ** stream) {
  return guard([&] {
    OnDevice on_dev(s);
    *stream = static_cast<void *>(s->st);
  });
}

rgpu_status rgpu_neighbour_list_build(rgpu_structures * s, double cutoff) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!(cutoff > 0)) throw Error(RGPU_ERR_INVALID_ARGUMENT, "cutoff must be > 0");
    build_nl(s, cutoff);
  });
}

rgpu_status rgpu_neighbour_list_size(const rgpu_structures * s, int64_t * n_centers, int64_t * n_pairs) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!s->nl_valid) throw Error(RGPU_ERR_NOT_COMPUTED, "the neighbour list has not been built");
    *n_centers = s->nl.n_centers;
    *n_pairs = s->nl.n_pairs;
  });
}

rgpu_status rgpu_neighbour_list_get(const rgpu_structures * s, int32_t * center_atom, int64_t * pair_offsets,
                                    int32_t * j_atom, int32_t * shift, double * distance, double * direction) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!s->nl_valid) throw Error(RGPU_ERR_NOT_COMPUTED, "the neighbour list has not been built");
    const int64_t nc = s->nl.n_centers, np = s->nl.n_pairs;
    auto get = [&](void * dst, const void * src, size_t bytes) {
      if (dst && bytes) RGPU_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->st));
    };
    get(center_atom, s->nl.center_atom, sizeof(int32_t) * nc);
    get(pair_offsets, s->nl.pair_off, sizeof(int64_t) * (nc + 1));
    get(j_atom, s->nl.pair_j, sizeof(int32_t) * np);
    get(shift, s->nl.pair_shift, sizeof(int32_t) * 3 * np);
    get(distance, s->nl.pair_dist, sizeof(double) * np);
    get(direction, s->nl.pair_dir, sizeof(double) * 3 * np);
    RGPU_CUDA(cudaStreamSynchronize(s->st));
  });
}

rgpu_status rgpu_compute(rgpu_calculator * calc, rgpu_structures * s, int precision, int gradients) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!calc || !s) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    if (precision != RGPU_PRECISION_FP64 && precision != RGPU_PRECISION_FP32)
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "unknown precision");
    bool g = gradients || calc->hy.compute_gradients;
    if (g && s->has_mask)
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "Can't compute spherical expansion gradients with masked center atoms",
                  RGPU_EXC_LOGIC_ERROR);
    calculator_to_device(calc);
    s->timed = false;
    compute_features(calc, s, precision, g, {});
    RGPU_CUDA(cudaStreamSynchronize(s->st));
  });
}

rgpu_status rgpu_get_species(const rgpu_structures * s, int32_t * n_species, int32_t * species) {
  return guard([&] {
    OnDevice on_dev(s);
    *n_species = int32_t(s->species.size());
    for (size_t i = 0; i < s->species.size(); ++i) species[i] = s->species[i];
  });
}

rgpu_status rgpu_get_feature_keys(const rgpu_calculator * calc, const rgpu_structures * s, int32_t * n_keys,
                                  int32_t * keys) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!s->feat_valid || s->feat_calc != calc) throw Error(RGPU_ERR_NOT_COMPUTED, "features have not been computed");
    auto k = present_keys(calc, s);
    *n_keys = int32_t(k.size());
    if (keys)
      for (size_t i = 0; i < k.size(); ++i) {
        keys[2 * i] = k[i].first;
        keys[2 * i + 1] = k[i].second;
      }
  });
}

rgpu_status rgpu_get_features(const rgpu_calculator * calc, const rgpu_structures * s, int32_t n_keys,
                              const int32_t * keys, double * out) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!s->feat_valid || s->feat_calc != calc) throw Error(RGPU_ERR_NOT_COMPUTED, "features have not been computed");
    const FeatureDims & fd = s->fd;
    const int64_t nc = s->nl.n_centers;
    const bool ps = calc->hy.kind == "sphericalinvariants";
    const int inner = ps ? fd.n * fd.n * (fd.L + 1) : fd.nK;
    const int row_len = ps ? fd.Dpad : fd.S * fd.nK;
    std::vector<int32_t> row_of(nc);
    RGPU_CUDA(cudaMemcpyAsync(row_of.data(), s->row_of_center.p, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, s->st));
    std::vector<double> dense(size_t(nc) * row_len);
    if (s->feat_precision == RGPU_PRECISION_FP64) {
      const void * src = ps ? s->X64.p : s->C64.p;
      RGPU_CUDA(cudaMemcpyAsync(dense.data(), src, sizeof(double) * dense.size(), cudaMemcpyDeviceToHost, s->st));
      RGPU_CUDA(cudaStreamSynchronize(s->st));
    } else {
      // FP32 expansion rows are padded ([S*n][row_stride(L)])
      const size_t rs = size_t(row_stride(fd.L));
      std::vector<float> tmp(ps ? size_t(nc) * fd.Dg : size_t(nc) * fd.S * fd.n * rs);
      const void * src = ps ? s->X32.p : s->C32.p;
      RGPU_CUDA(cudaMemcpyAsync(tmp.data(), src, sizeof(float) * tmp.size(), cudaMemcpyDeviceToHost, s->st));
      RGPU_CUDA(cudaStreamSynchronize(s->st));
      if (ps) {
        // FP32 rows hold the unnormalised p in the packed layout: scale by
        // 1/|p| and unfold into the reference's column order
        std::vector<float> scale(nc);
        RGPU_CUDA(cudaMemcpyAsync(scale.data(), s->xscale32.p, sizeof(float) * nc, cudaMemcpyDeviceToHost, s->st));
        RGPU_CUDA(cudaStreamSynchronize(s->st));
        for (int64_t r = 0; r < nc; ++r)
          unpack_to_reference(fd, &tmp[size_t(r) * fd.Dg], scale[r], &dense[size_t(r) * row_len]);
      } else {
        for (int64_t r = 0; r < nc; ++r)
          for (int row = 0; row < fd.S * fd.n; ++row)
            for (int l = 0; l <= fd.L; ++l)
              for (int m = 0; m < 2 * l + 1; ++m)
                dense[size_t(r) * row_len + size_t(row) * fd.K + l * l + m] =
                    tmp[(size_t(r) * fd.S * fd.n + row) * rs + offp(l) + m];
      }
    }
    auto blocks = key_blocks(calc, s, n_keys, keys);
    for (int64_t ci = 0; ci < nc; ++ci) {
      const double * src = &dense[size_t(ps ? row_of[ci] : ci) * row_len];
      double * dst = out + size_t(ci) * n_keys * inner;
      for (int k = 0; k < n_keys; ++k) {
        if (blocks[k] < 0)
          std::memset(dst + size_t(k) * inner, 0, sizeof(double) * inner);
        else
          std::memcpy(dst + size_t(k) * inner, src + size_t(blocks[k]) * inner, sizeof(double) * inner);
      }
    }
  });
}

rgpu_status rgpu_get_features_gradient(const rgpu_calculator * calc, const rgpu_structures * s_in, int32_t n_keys,
                                       const int32_t * keys, double * out) {
  return guard([&] {
    OnDevice on_dev(s_in);
    rgpu_structures * s = const_cast<rgpu_structures *>(s_in);
    if (!s->feat_valid || s->feat_calc != calc) throw Error(RGPU_ERR_NOT_COMPUTED, "features have not been computed");
    if (!s->feat_gradients) throw Error(RGPU_ERR_NOT_COMPUTED, "gradients were not requested (compute_gradients)");
    if (s->feat_precision != RGPU_PRECISION_FP64)
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "dense gradients are exported from the FP64 path");
    const FeatureDims & fd = s->fd;
    const int64_t nc = s->nl.n_centers;
    auto blocks = key_blocks(calc, s, n_keys, keys);
    if (calc->hy.kind == "sphericalexpansion") {
      export_expansion_gradient(calc, s, n_keys, blocks, out);
      return;
    }
    const int inner = fd.n * fd.n * (fd.L + 1);
    ExpansionArgs ea = exp_args(calc, s);
    PsArgs pa;
    pa.fd = fd;
    pa.n_centers = nc;
    pa.normalize = calc->hy.normalize;
    pa.row_of_center = s->row_of_center.as<int32_t>();
    const size_t per_pair = sizeof(double) * (3 * size_t(fd.D) + 3 * size_t(fd.nK));
    const size_t per_center = sizeof(double) * size_t(fd.S) * 3 * fd.nK;
    const size_t budget = size_t(4) << 30;
    std::vector<double> host;
    const std::vector<int64_t> & poff = pair_offsets_host(s);
    int64_t c0 = 0;
    while (c0 < nc) {
      int64_t c1 = c0;
      size_t bytes = 0;
      while (c1 < nc) {
        size_t add = per_pair * size_t(poff[c1 + 1] - poff[c1]) + per_center;
        if (c1 > c0 && bytes + add > budget) break;
        bytes += add;
        ++c1;
      }
      const int64_t p_base = poff[c0];
      const int64_t np = poff[c1] - p_base;
      s->dCp.ensure(sizeof(double) * size_t(np) * 3 * fd.nK + 64);
      s->dCs.ensure(per_center * size_t(c1 - c0) + 64);
      s->dXp.ensure(sizeof(double) * size_t(np) * 3 * fd.D + 64);
      launch_expansion_grad_fp64(ea, c0, c1, p_base, s->dCp.as<double>(), s->st);
      launch_expansion_selfgrad_fp64(ea, c0, c1, p_base, s->dCp.as<double>(), s->dCs.as<double>(), s->st);
      launch_ps_grad_fp64(pa, ea, c0, c1, p_base, s->C64.as<double>(), s->X64.as<double>(), s->invn64.as<double>(),
                          s->dCp.as<double>(), s->dCs.as<double>(), s->dXp.as<double>(), s->st);
      host.resize(size_t(np) * 3 * fd.D);
      RGPU_CUDA(cudaMemcpyAsync(host.data(), s->dXp.p, sizeof(double) * host.size(), cudaMemcpyDeviceToHost, s->st));
      RGPU_CUDA(cudaStreamSynchronize(s->st));
      for (int64_t p = 0; p < np; ++p)
        for (int c = 0; c < 3; ++c) {
          const double * src = &host[(size_t(p) * 3 + c) * fd.D];
          double * dst = out + (size_t(p_base + p) * 3 + c) * size_t(n_keys) * inner;
          for (int k = 0; k < n_keys; ++k) {
            if (blocks[k] < 0)
              std::memset(dst + size_t(k) * inner, 0, sizeof(double) * inner);
            else
              std::memcpy(dst + size_t(k) * inner, src + size_t(blocks[k]) * inner, sizeof(double) * inner);
          }
        }
      c0 = c1;
    }
  });
}

rgpu_status rgpu_gap_model_create(rgpu_calculator * calc, int32_t n_species, const int32_t * species,
                                  int32_t n_sparse, const int32_t * sparse_species, const double * T,
                                  const double * weights, int32_t zeta, const double * self_contributions,
                                  rgpu_gap_model ** out) {
  return guard([&] {
    if (!calc || !out || n_species <= 0 || n_sparse < 0) throw Error(RGPU_ERR_INVALID_ARGUMENT, "bad arguments");
    if (calc->hy.kind != "sphericalinvariants")
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "the GAP model needs a SphericalInvariants calculator");
    if (zeta < 1) throw Error(RGPU_ERR_INVALID_ARGUMENT, "zeta must be >= 1");
    auto m = std::make_unique<rgpu_gap_model>();
    m->calc = calc;
    m->species.assign(species, species + n_species);
    if (!std::is_sorted(m->species.begin(), m->species.end()))
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "model species must be sorted");
    m->M = n_sparse;
    m->sp_species.assign(sparse_species, sparse_species + n_sparse);
    for (int sp : m->sp_species)
      if (!std::binary_search(m->species.begin(), m->species.end(), sp))
        throw Error(RGPU_ERR_INVALID_ARGUMENT, "sparse point species missing from the model species");
    FeatureDims fm = make_dims(calc->hy, n_species);
    m->T.assign(T, T + size_t(n_sparse) * fm.D);
    if (weights)
      m->alpha.assign(weights, weights + n_sparse);
    else
      m->alpha.assign(size_t(n_sparse), 0.);  // kernel matrices only
    m->zeta = zeta;
    m->self_contrib.assign(n_species, 0.);
    if (self_contributions) m->self_contrib.assign(self_contributions, self_contributions + n_species);
    *out = m.release();
  });
}

rgpu_status rgpu_gap_model_destroy(rgpu_gap_model * m) {
  return guard([&] { delete m; });
}

rgpu_status rgpu_gap_predict(rgpu_gap_model * m, rgpu_structures * s, int precision, double * energies,
                             double * forces) {
  return guard([&] {
    OnDevice on_dev(s);
    gap_predict_entry(m, s, precision, energies, forces, nullptr);
  });
}

rgpu_status rgpu_gap_predict_stress(rgpu_gap_model * m, rgpu_structures * s, int precision, double * energies,
                                    double * forces, double * neg_stress) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!neg_stress) throw Error(RGPU_ERR_INVALID_ARGUMENT, "neg_stress output is required");
    gap_predict_entry(m, s, precision, energies, forces, neg_stress);
  });
}

rgpu_status rgpu_gap_forward_dev(rgpu_gap_model * m, rgpu_structures * s, const double * positions_dev,
                                 double * energies_dev) {
  return guard([&] {
    OnDevice on_dev(s);
    gap_forward_dev_impl(m, s, positions_dev, energies_dev);
  });
}

rgpu_status rgpu_gap_backward_dev(rgpu_gap_model * m, rgpu_structures * s, const double * energies_grad_dev,
                                  double * grad_dev) {
  return guard([&] {
    OnDevice on_dev(s);
    gap_backward_dev_impl(m, s, energies_grad_dev, grad_dev);
  });
}

rgpu_status rgpu_md_step(rgpu_gap_model * m, rgpu_structures * s, const double * positions, double * energies,
                         double * forces, double * neg_stress) {
  return guard([&] {
    OnDevice on_dev(s);
    md_step_impl(m, s, positions, energies, forces, neg_stress);
  });
}

rgpu_status rgpu_md_step_info(const rgpu_structures * s, int32_t * recorded, int64_t * info) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!s || !recorded) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    *recorded = s->md_exec ? 1 : 0;
    if (info) {
      info[0] = s->md_caps.sites;
      info[1] = s->md_caps.boxes;
      info[2] = s->md_caps.pairs;
      info[3] = s->md_replays;
      info[4] = s->md_reason;
      info[5] = s->md_kernels;
    }
  });
}

rgpu_status rgpu_sparse_kernel(rgpu_gap_model * m, rgpu_structures * s, int32_t target_atom, double * out) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!out) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    sparse_kernel_impl(m, s, target_atom != 0, out);
  });
}

rgpu_status rgpu_sparse_kernel_derivative(rgpu_gap_model * m, rgpu_structures * s, int32_t neg_stress,
                                          double * out) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!out) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    sparse_kernel_derivative_impl(m, s, neg_stress != 0, out);
  });
}

rgpu_status rgpu_sparse_kernel_mm(rgpu_gap_model * m, double * out) {
  return guard([&] {
    if (!out) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    sparse_kernel_mm_impl(m, out);
  });
}

namespace {
__global__ void bf16_pair_to_f32_kernel(const __nv_bfloat16 * hi, const __nv_bfloat16 * lo, int64_t rows,
                                        int64_t cols, int64_t ld, float * out) {
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  int64_t r = i / cols, c = i - r * cols;
  out[i] = __bfloat162float(hi[r * ld + c]) + __bfloat162float(lo[r * ld + c]);
}
__global__ void sum_parts_kernel(const float * parts, int n_parts, int64_t M, float * e) {
  int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= M) return;
  float s = 0.f;
  for (int t = 0; t < n_parts; ++t) s += parts[int64_t(t) * M + r];
  e[r] = s;
}
}  // namespace

// Scratch of the GEMM test hook, one set per device (the hook is called
// from one host thread at a time).
struct DebugGemmBuffers {
  DevBuf ah, al, bh, bl, wh, wl, parts;
};
static PerDevice<DebugGemmBuffers> g_debug_gemm_buffers;

rgpu_status rgpu_debug_set_gemm_wait_limit(int64_t polls) {
  return guard([&] { set_gemm_wait_limit(polls); });
}

rgpu_status rgpu_debug_packed_layout(int32_t S, int32_t max_radial, int32_t max_angular, int64_t * D, int64_t * Dg,
                                     const double * ref, double * packed, double * unpacked) {
  return guard([&] {
    if (S < 1 || S > kMaxSpecies || max_radial < 1 || max_angular < 0 || max_angular > kMaxL)
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "bad layout shape");
    Hypers hy;
    hy.max_radial = max_radial;
    hy.max_angular = max_angular;
    const FeatureDims fd = make_dims(hy, S);
    if (D) *D = fd.D;
    if (Dg) *Dg = fd.Dg;
    if (!ref) return;
    std::vector<double> pk(fd.Dg);
    pack_reference_row(fd, ref, pk.data());
    if (packed) std::copy(pk.begin(), pk.end(), packed);
    if (unpacked) {
      std::vector<float> pf(pk.begin(), pk.end());
      unpack_to_reference(fd, pf.data(), 1.f, unpacked);
    }
  });
}

rgpu_status rgpu_debug_gemm_bf16x3(int mode, int64_t M, int64_t N, int64_t K, const float * A, const float * B,
                                   const float * alpha, int32_t zeta, float * C, float * e, void * stream) {
  return guard([&] {
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) throw Error(RGPU_ERR_INVALID_ARGUMENT, "bad GEMM arguments");
    if (mode == 0 && N % 4 != 0) throw Error(RGPU_ERR_INVALID_ARGUMENT, "N must be a multiple of 4");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DebugGemmBuffers & B_ = g_debug_gemm_buffers.at(current_device());
    DevBuf &ah = B_.ah, &al = B_.al, &bh = B_.bh, &bl = B_.bl, &wh = B_.wh, &wl = B_.wl, &parts = B_.parts;
    const int64_t Kp = (K + 63) / 64 * 64, Np = (N + 31) / 32 * 32;
    ah.ensure(2 * size_t(M) * Kp);
    al.ensure(2 * size_t(M) * Kp);
    bh.ensure(2 * size_t(N) * Kp);
    bl.ensure(2 * size_t(N) * Kp);
    split_bf16(A, M, K, K, ah.as<__nv_bfloat16>(), al.as<__nv_bfloat16>(), Kp, st);
    split_bf16(B, N, K, K, bh.as<__nv_bfloat16>(), bl.as<__nv_bfloat16>(), Kp, st);
    Bf16x3Gemm g{};
    g.M = M;
    g.N = N;
    g.K = Kp;
    g.A_hi = ah.as<__nv_bfloat16>();
    g.A_lo = al.as<__nv_bfloat16>();
    g.lda = Kp;
    g.B_hi = bh.as<__nv_bfloat16>();
    g.B_lo = bl.as<__nv_bfloat16>();
    g.ldb = Kp;
    g.epilogue = mode;
    if (mode == 0) {
      g.C = C;
      g.ldc = N;
      gemm_bf16x3(g, st);
    } else {
      const int n_parts = int((N + kTcTileN - 1) / kTcTileN);
      wh.ensure(2 * size_t(M) * Np);
      wl.ensure(2 * size_t(M) * Np);
      parts.ensure(sizeof(float) * size_t(n_parts) * M);
      g.W_hi = wh.as<__nv_bfloat16>();
      g.W_lo = wl.as<__nv_bfloat16>();
      g.ldw = Np;
      g.alpha = alpha;
      g.zeta = zeta;
      g.e_part = parts.as<float>();
      gemm_bf16x3(g, st);
      bf16_pair_to_f32_kernel<<<div_up(M * N, 256), 256, 0, st>>>(g.W_hi, g.W_lo, M, N, Np, C);
      if (e) sum_parts_kernel<<<div_up(M, 256), 256, 0, st>>>(parts.as<float>(), n_parts, M, e);
    }
    RGPU_CUDA(cudaStreamSynchronize(st));
    const int where = gemm_tc_timeout(true);
    if (where) throw Error(RGPU_ERR_TIMEOUT, "tensor-core GEMM wait gave up at stage " + std::to_string(where));
  });
}

rgpu_status rgpu_gap_energies_noalloc(int64_t M, int64_t N, int64_t K, const float * A, const float * B,
                                      const float * alpha, int32_t zeta, float * e, void * stream) {
  return guard([&] { gap_energies_noalloc(M, N, K, A, B, alpha, zeta, e, static_cast<cudaStream_t>(stream)); });
}

rgpu_status rgpu_set_tile_config(int32_t n_species, int32_t max_radial, int32_t max_angular, const int32_t * values,
                                 int32_t n_values) {
  return guard([&] {
    if (n_values == 0) {
      set_tile_config(n_species, max_radial, max_angular, nullptr);
      return;
    }
    if (n_values != kTileFields || !values)
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "tile config: " + std::to_string(kTileFields) + " values expected");
    const TileConfig c = tile_config_from_array(values);
    set_tile_config(n_species, max_radial, max_angular, &c);
  });
}

rgpu_status rgpu_get_tile_config(int32_t n_species, int32_t max_radial, int32_t max_angular, int32_t * values) {
  return guard([&] {
    if (!values) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    tile_config_to_array(tile_config(n_species, max_radial, max_angular), values);
  });
}

rgpu_status rgpu_structures_use_graphs(rgpu_structures * s, int enable) {
  return guard([&] {
    OnDevice on_dev(s);
    if (!s) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    s->use_graphs = enable != 0;
    if (!s->use_graphs) {
      RGPU_CUDA(cudaStreamSynchronize(s->st));
      for (PredictGraph & g : s->pgraphs) pgraph_release(g);
      s->pgraphs.clear();
    }
  });
}

rgpu_status rgpu_structures_graph_info(const rgpu_structures * s, int64_t * info) {
  return guard([&] {
    if (!s || !info) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    info[0] = int64_t(s->pgraphs.size());
    info[1] = s->pgraph_replays;
    info[2] = s->pgraph_records;
    info[3] = s->pgraph_last_kernels;
  });
}

rgpu_status rgpu_measure_fma_peak(int precision, double * tflops) {
  return guard([&] {
    if (!tflops) throw Error(RGPU_ERR_INVALID_ARGUMENT, "null argument");
    if (precision != RGPU_PRECISION_FP64 && precision != RGPU_PRECISION_FP32)
      throw Error(RGPU_ERR_INVALID_ARGUMENT, "unknown precision");
    *tflops = measure_fma_peak(precision);
  });
}

rgpu_status rgpu_synchronize(rgpu_structures * s) {
  return guard([&] {
    OnDevice on_dev(s);
    RGPU_CUDA(cudaStreamSynchronize(s->st));
  });
}

int64_t rgpu_kernel_launches(int reset) { return rgpu::launches(reset != 0); }

rgpu_status rgpu_stage_times(const rgpu_structures * s, double * ms_out, int32_t n_stages) {
  return guard([&] {
    OnDevice on_dev(s);
    RGPU_CUDA(cudaStreamSynchronize(s->st));
    // 0 whole call, 1 neighbour list, 2 expansion, 3 power spectrum,
    // 4 forward GEMMs, 5 backward GEMMs, 6 power-spectrum backward (plain:
    // gradient chunks), 7 pair adjoint
    const int pairs[8][2] = {{0, 8}, {0, 1}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}, {7, 8}};
    for (int i = 0; i < n_stages && i < 8; ++i) {
      float ms = 0.f;
      cudaError_t e = cudaEventElapsedTime(&ms, s->ev[pairs[i][0]], s->ev[pairs[i][1]]);
      ms_out[i] = (e == cudaSuccess) ? ms : -1.0;
    }
  });
}

}  // extern "C"
