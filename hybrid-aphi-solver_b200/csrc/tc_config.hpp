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
constexpr int kTcPlanes = 10;    // pre-split operand planes per stage: A re/im x hi/lo, B (-Bi, Br, Bi) x hi/lo
constexpr int kTcPlaneA = kTcM * kTcK * 4;      // bytes of one A plane in one stage
constexpr int kTcPlaneB = kTcN * kTcK * 4;      // bytes of one B plane in one stage
// Bytes of one split-operand stage, and the dynamic shared memory of a tile,
// for a split into `Split` TF32 planes.
// The two-piece split stacks its B planes (-Bi, Br, Bi per piece) so that
// the complex product needs two M128 N128 MMAs per kept pair; the
// three-piece split keeps separate Br, Bi planes and four M128 N64 MMAs (its
// stacked form would not leave room for two CTAs per SM).
template <int Split>
struct TcLayout {
    static constexpr bool stacked = Split == 2;
    static constexpr int b_planes = stacked ? 3 : 2;  // B planes per piece
};
template <int Split>
struct TcBytes {
    static constexpr int stage = 2 * Split * kTcPlaneA + TcLayout<Split>::b_planes * Split * kTcPlaneB;
};
constexpr int kTcStage = TcBytes<kTcSplit>::stage;
constexpr int kTcRawA = kTcK * kTcM * 8;        // complex64 A rows of one stage
constexpr int kTcRawB = kTcK * kTcN * 8;
constexpr int kTcRawStage = kTcRawA + kTcRawB + kTcK * 8;  // + the stage's pivots
constexpr int kTcTmemCols = 4 * kTcN;           // Cr, Ci main + Cr, Ci corrections
template <int Split, int Stages = kTcPlaneStages>
struct TcSmem {
    static constexpr int bytes = Stages * TcBytes<Split>::stage + kTcRawStages * kTcRawStage + 64;
};
constexpr int kTcSmem = TcSmem<kTcSplit>::bytes;

}  // namespace aphi_b200
