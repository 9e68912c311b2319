// pmp_handle.h -- the library's private handle (struct pmp_spray) and the
// helpers shared by its translation units.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "phys/pmp_thermo.h"
#include "pmp_device.cuh"

namespace pmp {

constexpr int kBlock = 128;
constexpr int kSortPad = 8;  // cells of margin in the sort key around a box

struct BoxStore {
  long long n = 0;
  double* d = nullptr;  // (3 + NR) * n doubles, sorted by cell
  int* id = nullptr;
  long long* perm = nullptr;  // sorted slot -> caller index
};

struct LearnState;  // learned form (pmp_learn.cu)

// A device copy of one update call's box table (a BoxEntry per box).  Calls
// reuse the slot whose content they repeat, so the steady state uploads
// nothing; a new table is uploaded from the slot's page-locked staging on the
// call's stream.  A slot read by a captured CUDA graph is held (never
// rewritten) while that graph exists.
struct TableSlot {
  std::vector<BoxEntry> host;      // the table's content
  BoxEntry* d = nullptr;           // device copy
  BoxEntry* stage = nullptr;       // page-locked staging of the upload
  int cap = 0;
  cudaEvent_t uploaded = nullptr;  // completion of the last upload
  cudaStream_t stream = nullptr;   // the stream that upload was issued on
  unsigned long long last_use = 0;
  int holds = 0;                   // captured graphs that read this slot
};
constexpr int kTableSlots = 8;

// (box, first slot) work items of `chunk` slots (batched form, pmp_batch.cu)
struct WorkMap {
  int chunk = 0;
  int nitems = 0;
  int* box = nullptr;
  long long* start = nullptr;
  std::vector<int> item_begin;  // per box: first work item (nboxes + 1 entries)
};

struct BatchState {
  pmp_launch_config cfg{PMP_LAUNCH_GRID, 128, 96, 512, 0, 0};
  std::vector<WorkMap> maps;
  int* d_counter = nullptr;
  int sm_count = 0;
  // resident CTAs of the persistent launch, for the shape occ_cfg
  pmp_launch_config occ_cfg{-1, 0, 0, 0, 0, 0};
  int occ_ns = 0, occ_nf = 0;
  int persist_ctas = 0;
  // CUDA graphs of recent updates' device work (a few, so that alternating
  // calls such as MKD and MK both replay), least recently used evicted
  struct Graph {
    std::vector<unsigned char> key;
    cudaGraphExec_t exec = nullptr;
    unsigned long long last_use = 0;
    int table_slot = -1;  // the box-table slot the graph reads (held)
  };
  std::vector<Graph> graphs;
  unsigned long long use_clock = 0;
  cudaStream_t gstream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
};

}  // namespace pmp

struct pmp_spray {
  int device = 0;
  int nfuel = 0;
  int nspec = 0;
  char species[PMP_MAX_SPEC][PMP_NAME_LEN];
  pmp_mech mech;
  pmp_spray_data data;
  bool have_data = false;
  pmp_spray_comps comps;
  bool have_comps = false;
  pmp_geometry geom;
  bool have_geom = false;
  std::vector<pmp_box> boxes;
  int mode = PMP_MODE_FP64;
  int pelec = 0;  // enum pmp_coupling
  pmp::DevMech dmech;
  pmp::DevFuel dfuel;
  pmp::DevMechF dmechf;
  int spec_perm[PMP_MAX_SPEC];  // species order of dmechf (see DevMechF)
  int fuel_first = 0;
  pmp::DevFuelF dfuelf;
  // per-box staged droplets (before packing)
  std::vector<pmp::BoxStore> staged;
  std::vector<bool> box_set;
  // packed droplets
  bool packed = false;
  long long total = 0;
  double* soa = nullptr;  // (3 + NR) arrays of length total
  int* ids = nullptr;
  long long* perm = nullptr;
  std::vector<long long> box_begin;
  int ncta = 0;
  int cta_cap = 0;  // allocated entries of d_cta_box / d_cta_start
  int* d_cta_box = nullptr;
  long long* d_cta_start = nullptr;
  long long* d_box_begin = nullptr;
  long long* fb_list = nullptr;  // fallback slots (mixed / learned forms)
  pmp::BoxEntry* h_boxes = nullptr;  // the box table of the call being prepared
  int boxes_cap = 0;
  pmp::TableSlot tables[pmp::kTableSlots];
  unsigned long long table_clock = 0;
  int cur_table = -1;  // slot of the last prepared call's table
  pmp::DevStatus* d_status = nullptr;
  pmp::DevStatus* h_status = nullptr;
  // the first device error code, written by the kernels into page-locked
  // host memory mapped into the device (err_dev: its device address)
  int* err_host = nullptr;
  int* err_dev = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // stream-ordered updates: the stream of the last call and an event after
  // its device work; pending = work enqueued since the last pmp_spray_sync
  cudaStream_t last_stream = nullptr;
  cudaEvent_t ev_done = nullptr;
  bool pending = false;
  // the mixed form's FP64 list kernel runs on `side` beside the mixed kernel
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_sel = nullptr;
  pmp_error_info last_err;
  pmp_stats stats;
  // view pointers already checked to be device-accessible
  std::vector<const double*> checked_state, checked_src;
  // device mirrors of host views for pmp_spray_update_host
  std::vector<double*> stage_state, stage_src;
  std::vector<size_t> stage_state_n, stage_src_n;
  // pmp_spray_set_host_source_in: 1 = the host source is copied in and the
  // deposits added to it, 0 = it is taken as zero (device mirror cleared)
  int host_src_in = 1;
  // streams and events of the overlapped host-view update (copy-in, copy-out;
  // per stage: copied in, updated; start; all copied out)
  static constexpr int kHostStages = 8;
  cudaStream_t hs_in = nullptr, hs_out = nullptr;
  cudaEvent_t hev_in[kHostStages] = {}, hev_done[kHostStages] = {};
  cudaEvent_t hev_start = nullptr, hev_out = nullptr;
  pmp::LearnState* learn = nullptr;
  pmp::BatchState batch;
  // cell -> box map over the domain (pmp_mesh.cu), rebuilt when the grids or
  // the geometry change
  int grids_version = 0;
  int box_map_version = -1;
  int* d_box_map = nullptr;
  void* mesh_scratch = nullptr;
  size_t mesh_scratch_bytes = 0;
  // re-binning (pmp_spray_redistribute): its working arrays (sort keys and
  // values, CUB's temporary storage), kept between calls, and a spare
  // droplet store that the re-binned droplets are gathered into (the old
  // store then becomes the spare); spare_cap droplets
  void* rebin_scratch = nullptr;
  size_t rebin_scratch_bytes = 0;
  double* soa_spare = nullptr;
  int* ids_spare = nullptr;
  long long spare_cap = 0;
  // gas records of the grown boxes (BoxEntry::gr, FP32, mixed and learned
  // forms; BoxEntry::gr64, FP64 form): capacity in bytes, and the largest
  // grown box (cells) of the last prepared update
  void* gas_rec = nullptr;
  size_t gas_rec_bytes = 0;
  int gas_rec_max_cells = 0;
  int nr() const { return PMP_PSTATE_NUM(nfuel); }
  int ncomp() const { return 3 + nr(); }
};

namespace pmp {

// pmp_spray.cu
int set_err(pmp_spray* h, int code, const char* msg, int box = -1, long long particle = -1);
// wait for the handle's enqueued update work (entry points that read or
// replace the droplets, or free buffers the kernels use, call it first)
void quiesce(pmp_spray* h);
// read, report and clear the device status after the handle's last call
// (pmp_spray_sync): the first device error of the calls since the previous
// sync, or PMP_OK; fills stats and the error record
int sync_status(pmp_spray* h);
// release a box-table slot held by a captured graph
void release_table(pmp_spray* h, int slot);
// validate views, pack droplets, upload the box table, reset the status
// block and fill the kernel parameters of one update call
int prepare_update(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes,
  double flow_dt, int state_ghosts, int source_ghosts, int is_ghost, int do_move,
  double spray_cfl_lev, cudaStream_t st, KParams& P);
int run_fp64_list(int ns, int nf, const KParams& P, long long total, cudaStream_t st);
int dispatch_fp64_default(int ns, int nf, const KParams& P, int ncta, cudaStream_t st);
// the device work of one update after prepare: the per-call fallback count
// reset, timing events, kernels (no synchronisation, no status read-back)
int enqueue_update(pmp_spray* h, const KParams& P, int nboxes, cudaStream_t st);
// a whole update call, synchronous (prepare, launch, sync_status)
int run_update(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes,
  double flow_dt, int state_ghosts, int source_ghosts, int is_ghost, int do_move,
  double spray_cfl_lev, cudaStream_t st);
// pack the staged droplets if needed
int ensure_packed(pmp_spray* h);
// after re-binning: the store (soa, ids, perm) already holds the droplets in
// their new order; install the new box bounds and rebuild the CTA map
int install_rebinned(pmp_spray* h, const std::vector<long long>& box_begin);
// pmp_mesh.cu
void mesh_free(pmp_spray* h);
// pmp_batch.cu
int batch_enqueue_fp64(pmp_spray* h, const KParams& P, int nboxes, cudaStream_t st);
// FP64 gas records (BoxEntry::gr64) of boxes [b0, b0 + nb), the handle's coupling;
// a no-op when the update runs without them
int launch_gas_records64(const pmp_spray* h, const KParams& P, int b0, int nb, cudaStream_t st);
int graph_update(pmp_spray* h, const KParams& P, int nboxes, cudaStream_t st, int* graph_state);
void batch_reset(pmp_spray* h);
void batch_free(pmp_spray* h);
// pmp_learn.cu
// the learned kernel over CTA-map items [first, first + count) (count < 0: all);
// the audit runs only with the whole map
int launch_learned(pmp_spray* h, const KParams& P, cudaStream_t st, int first = 0, int count = -1);
bool learn_audit_on(const pmp_spray* h);
bool learn_ready(const pmp_spray* h);
void learn_free(pmp_spray* h);

}  // namespace pmp
