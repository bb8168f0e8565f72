// Schedule autotuner: for each tunable decision of the engine and each
// (matrix order, batch size class) it keeps the choice that ran fastest when
// timed on this GPU.  Decisions:
//   kTuneLU       LU factorisation schedule (0: one CTA per matrix, 1: panel
//                 by panel over all SMs)
//   kTuneSchur    Schur crossover: active blocks below it use single-shift
//                 sweeps, larger ones multishift sweeps with early deflation
//   kTuneProduct  cascade products of mixed plans and their tile shape
//                 (0: 3xTF32 on tcgen05, 128 x 128 tiles; 1: FP64 tensor path;
//                 2: 3xTF32 on tcgen05, 128 x 256 tiles)
// The table is host data (thread-safe); measuring needs the engine's device.
#pragma once
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"

struct rcwa_engine;

enum TuneOp { kTuneLU = 0, kTuneSchur = 1, kTuneProduct = 2, kTuneOps = 3 };
constexpr int kTuneMaxCand = 4;

// modes of an engine's tuner
enum TuneMode { kTuningOff = 0, kTuningTable = 1, kTuningAuto = 2 };

struct TuneEntry {
  int choice = -1;
  int ncand = 0;
  int cand[kTuneMaxCand] = {};
  double ms[kTuneMaxCand] = {};  // time of each candidate (0: not measured)
};

struct rcwa_tuner {
  int sms = 148;
  std::map<std::tuple<int, int, int>, TuneEntry> table;  // (op, n, batch class)
  mutable std::mutex mu;
};

// Batch size class: the number of waves of one-CTA-per-matrix work, 1, 2, 3,
// 4 (4..7 waves) or 8 (8 and more).
int tune_batch_class(int batch, int sms);
// Candidate choices of a decision at order n; returns their count.
int tune_candidates(int op, int n, int* out);
// The built-in rule, used when the table has no entry and measuring is off.
int tune_default(int op, int n, int batch);
// The same rule for a given SM count (sms <= 0: this device's).
int tune_default_sms(int op, int n, int batch, int sms);
// The choice the engine uses for (op, n, batch): its tuner's entry, else a
// fresh measurement (automatic mode), else the built-in rule.  Host code
// outside stream capture only (a measurement synchronises the engine stream).
int tune_resolve(rcwa_engine* e, int op, int n, int batch);
// Times every candidate of (op, n, batch) on synthetic inputs on the engine's
// stream and fills `out` (choice = the fastest).  Inputs: seeded random
// matrices; LU and products at the given batch (capped by memory), the
// eigensolver on one wave of matrices.
cudaError_t tune_measure(rcwa_engine* e, int op, int n, int batch, TuneEntry& out);
