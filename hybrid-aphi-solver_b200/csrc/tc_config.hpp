// Shapes of the tensor-core update (tc_update.cuh), shared with the host-side
// planner.
#pragma once

namespace aphi_b200 {

constexpr int kTcM = 128;        // complex rows per tile
constexpr int kTcN = 64;         // complex columns per tile
constexpr int kTcK = 8;          // K per pipeline stage (one MMA step)
constexpr int kTcPlaneStages = 2;  // split-operand stages the tensor core reads
constexpr int kTcRawStages = 3;  // raw-operand stages in flight (cp.async, two ahead)
constexpr int kTcGroup = 2;      // stages per fresh main accumulator (then drained to registers)
constexpr int kTcSplit = 3;      // default: x = hi + mid + lo, each TF32 (2: x ~ hi + lo)
constexpr int kTcPanel = 128;    // panel width whose trailing update goes to the tensor cores
constexpr int kTcThreads = 128;
constexpr int kTcPlaneA = kTcM * kTcK * 4;      // bytes of one A plane in one stage
constexpr int kTcPlaneB = kTcN * kTcK * 4;      // bytes of one B plane in one stage
// Bytes of one split-operand stage, and the dynamic shared memory of a tile,
// for a split into `Split` TF32 planes.
template <int Split>
struct TcBytes {
    static constexpr int stage = 2 * Split * (kTcPlaneA + kTcPlaneB);
};
constexpr int kTcStage = TcBytes<kTcSplit>::stage;
constexpr int kTcRawA = kTcK * kTcM * 8;        // complex64 A rows of one stage
constexpr int kTcRawB = kTcK * kTcN * 8;
constexpr int kTcRawStage = kTcRawA + kTcRawB + kTcK * 8;  // + the stage's pivots
constexpr int kTcTmemCols = 4 * kTcN;           // Cr, Ci main + Cr, Ci corrections
template <int Split>
struct TcSmem {
    static constexpr int bytes = kTcPlaneStages * TcBytes<Split>::stage + kTcRawStages * kTcRawStage + 64;
};
constexpr int kTcSmem = TcSmem<kTcSplit>::bytes;

}  // namespace aphi_b200
