// Device-side analysis: the supernodal schedule uploaded once per pattern,
// plus the launch plans (work lists per elimination-tree level) that the
// numeric factorization and the solves replay.
#pragma once

#include "tc_config.hpp"

#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "aphi_b200.h"
#include "symbolic.hpp"

namespace aphi_b200 {

// Work item kinds.
enum Kind : int {
    K_EXTEND_ADD = 0,  // (s, col0): zero CB columns, add children's CBs, for 32 front columns
    K_SMALL = 1,       // (s): whole front in shared memory
    K_DIAG = 2,        // (s, k0): factor the diagonal block of step k0
    K_TRSM = 3,        // (s, k0, row0): rows row0.. of L21 for step k0
    K_UPDATE_WIDE = 4,  // (s, p0, i0, j0): SIMT trailing update by a whole panel
    K_FWD_GATHER = 5,  // (s): children's update vectors into the front vector
    K_FWD_DIAG = 6,    // (s, blk): unit-triangle solve of a 64-column block
    K_FWD_UPDATE = 7,  // (s, blk, row0): rows below the block
    K_BWD_UPDATE = 8,  // (s, blk, row0, slot): partial L^T x sums over a row chunk
    K_BWD_DIAG = 9,    // (s, blk, first slot, slots): block of the transposed solve
    K_UPDATE_PANEL = 10,  // (s, k0, i0, j0): update tile restricted to the current 128-column panel
    K_UPDATE_TC = 11,     // (s, p0, i0, j0, d): tensor-core trailing update by a whole panel
    K_TC_SPLIT = 12,      // (s, p0, r0, d): a front's trailing operands split into TF32 planes, 128 rows
    K_DMMA_SCALE = 13,    // (s, p0, r0, d): a front's trailing rows scaled by the group's pivots (W = L D), 128 rows
};

struct Launch {
    int kind;
    long long first;  // offset into the item array
    int count;
    int kcap = kTcPanel;  // trailing updates: panel columns applied at once (K = min(kcap, w - p0))
    int wide = 0;         // K_UPDATE_PANEL: 128 x 64 tiles on the trailing-update kernels (column cap at the panel's end);
                          // K_FWD_GATHER / K_FWD_UPDATE / K_BWD_UPDATE: fused with the triangle solve (see build_plans)
};

struct Item {
    int s, a, b, c;
    int d = 0;  // staged trailing updates and their operand launches: the front's region, in 256-byte units
                // of an entry's workspace (K_UPDATE_TC / K_TC_SPLIT; K_UPDATE_WIDE / K_DMMA_SCALE)
};

constexpr int kStep = 32;        // pivot block width of the blocked factorization
constexpr int kTile = 64;        // update tile
constexpr int kTrsmRows = 128;   // rows per TRSM block
constexpr int kPanelGroup = 4;                 // most panels per trailing update of the rest of a front
constexpr int kWidePair = kPanelGroup * kTcPanel;  // the most panel columns one trailing update applies
// Fronts this tall group 4 panels, smaller ones 2. A build may lower the
// threshold (the host-side plan checker does, to reach 4-panel groups on
// fronts small enough to replay on a CPU).
#ifndef APHI_GROUP4_ROWS
#define APHI_GROUP4_ROWS 8192
#endif
constexpr int kGroup4Rows = APHI_GROUP4_ROWS;
constexpr int kEaCols = 32;      // front columns per extend-add item
constexpr int kSolveBlock = 64;  // columns per triangular-solve block
constexpr int kSolveRows = 64;   // rows per solve update item

struct DeviceSchedule {
    int* first = nullptr;
    int* rows = nullptr;
    long long* loff = nullptr;
    long long* cboff = nullptr;
    long long* soff = nullptr;
    int* structs = nullptr;
    long long* reloff = nullptr;
    int* rel = nullptr;
    int* child_ptr = nullptr;
    int* child_list = nullptr;
    long long* uoff = nullptr;  // update-vector offsets (solve), per supernode
    long long* a_dest = nullptr;
    int* row_ptr = nullptr;     // upper CSR, original numbering
    int* col_idx = nullptr;
    int* new_of_orig = nullptr;
    int* orig_of_new = nullptr;
    int* ref_of_post = nullptr;
    int* fptr = nullptr;        // both triangles of A: row pointers,
    int* fcol = nullptr;        // columns,
    long long* fmap = nullptr;  // and the index of each entry in the upper values
    Item* items = nullptr;
};

}  // namespace aphi_b200

struct aphi_analysis {
    aphi_b200::Symbolic S;
    aphi_analysis_options opt{};
    aphi_b200::DeviceSchedule d;
    std::vector<aphi_b200::Launch> plan_factor, plan_factor_tc, plan_fwd, plan_bwd;
    std::vector<aphi_b200::Launch> plan_fwd_split, plan_bwd_split;  // the same solves, triangles as launches of their own
    std::vector<aphi_b200::Item> h_items;
    std::vector<long long> h_uoff;
    std::vector<int> h_row_ptr, h_col_idx;
    std::vector<int> h_fptr, h_fcol;
    std::vector<long long> h_fmap;
    bool on_device = false;
    int device = -1;       // the CUDA device holding the device copy (set with it)
    bool fronts = false;   // built from independent dense fronts (no matrix pattern)
    // Contribution-block workspaces shared by this analysis's factors, one per
    // precision ([0] FP64, [1] FP32), so that an FP64 and an FP32
    // factorization can run at the same time on different streams; each is
    // held by its lock while a factorization (or aphi_fronts_read) uses it.
    void* ws[2] = {nullptr, nullptr};
    size_t ws_bytes[2] = {0, 0};
    std::mutex ws_mu[2];
    long long num_items = 0;
    long long upool = 0;   // update-vector pool entries (per rhs)
    int max_parts = 1;
    long long stat_first = 0;  // items of the statistics pass (s, col0)
    int stat_count = 0;     // partial-sum slots of the largest backward update launch
    long long tc_ws_units = 0;    // split-operand workspace of the tensor-core plan, per entry (256-byte units)
    long long dmma_ws_units = 0;  // scaled-operand (W = L D) workspace of the FP64 plan, per entry (256-byte units)
    long long device_bytes = 0;
    ~aphi_analysis();
};

namespace aphi_b200 {
aphi_analysis* analysis_create(int n, const int* row_ptr, const int* col_idx, const int* perm,
                               const int* parent, const int* col_count, const aphi_analysis_options& o);
aphi_analysis* analysis_create_fronts(int count, const int* rows, const int* widths, const aphi_analysis_options& o);
void analysis_destroy(aphi_analysis* a);
void analysis_ensure_device(aphi_analysis* a);
void analysis_info(const aphi_analysis* a, double* info);
const Symbolic& analysis_symbolic(const aphi_analysis* a);
}  // namespace aphi_b200
