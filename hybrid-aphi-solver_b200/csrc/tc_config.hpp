// Shapes of the tensor-core update (tc_update.cuh), shared with the host-side
// planner.
#pragma once

namespace aphi_b200 {

constexpr int kTcM = 128;        // complex rows per tile
constexpr int kTcN = 64;         // complex columns per tile
constexpr int kTcK = 8;          // K per pipeline stage (one MMA step)
constexpr int kTcStages = 3;     // shared-memory stages in flight
constexpr int kTcSplit = 3;      // x = hi + mid + lo, each TF32
constexpr int kTcPanel = 128;    // panel width whose trailing update goes to the tensor cores
constexpr int kTcThreads = 128;
constexpr int kTcPlaneA = kTcM * kTcK * 4;      // bytes of one A plane in one stage
constexpr int kTcPlaneB = kTcN * kTcK * 4;      // bytes of one B plane in one stage
constexpr int kTcStage = 2 * kTcSplit * (kTcPlaneA + kTcPlaneB);
constexpr int kTcTmemCols = 4 * kTcN;           // Cr, Ci main + Cr, Ci corrections
constexpr int kTcSmem = kTcStages * kTcStage + 64;

}  // namespace aphi_b200
