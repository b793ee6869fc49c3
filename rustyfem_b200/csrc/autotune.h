// Autotuner of the plan's small-front / large-front cutover and tile shape.
//
// The outer Schur update of a front uses 64×64 tiles on the CUDA cores while its
// trailing matrix is small and 128-row tiles (tensor cores in the mixed path,
// k_schur_dmma in FP64) from Tuning::big_min_rows trailing rows on; on the tensor
// cores those tiles are 128×256 or 128×128 (Tuning::outer_tn). Where the crossover
// lies and which tile shape wins depend on the device, the precision and the shape
// of the tree, so the tuner measures them: for each candidate (cutover, tile width)
// it builds the plan and an engine, runs the numeric phase on the caller's values
// (the first run launches directly, the next two replay the captured graph) and keeps
// the candidate with the shortest device time. Cutovers that give the same tile split
// as an earlier one are not re-measured. Results are cached per (device, precision,
// tensor cores, symbolic analysis) for the life of the process.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <vector>

#include "engine.h"
#include "plan.h"
#include "symbolic.h"

namespace rfg {

struct TuneResult {
    Tuning best;
    std::vector<int64_t> cutover;  // candidates measured, in order: cutover rows
    std::vector<int64_t> tile_n;   //   and tensor-core outer-update tile width
    std::vector<double> ms;        // their numeric-phase device time (best of two replays)
    bool cached = false;           // taken from an earlier tuning of the same analysis
};

// make_engine builds the engine of a candidate plan (with the scatter of the original
// entries, which depends on the plan's layout). src: the caller's values (host).
// Returns the default tuning, unmeasured, when a candidate's factorization reports a
// failing pivot.
TuneResult autotune_cutover(const Symbolic& S, const std::function<std::unique_ptr<Engine>(Plan&&)>& make_engine,
                            const double* src, Precision prec, bool use_tc, const Tuning& base = Tuning());

}  // namespace rfg
