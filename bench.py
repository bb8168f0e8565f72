#!/usr/bin/env python
"""Throughput benchmark: RCWA solves/s on B200.

Workload (default): the 2D rectangular-pillar grating, Nx=Ny=10 (441 orders,
882 x 882 complex layer matrices), period 400 x 400 nm, 5 patterned layers,
256 wavelengths x 8 conical incidences (2048 solves), seeded synthetic inputs.
One step = one batched pass of the full RCWA solve (convolution matrices,
per-layer eigenproblems, interface solves, S-matrix cascade, per-order
efficiencies of TE and TM) over a batch of --batch points of that sweep.

value: the mixed-precision engine (cascade products in 3xTF32 on the tcgen05
tensor cores, everything else FP64): device time of K plan executions with the
inputs resident (CUDA events on the launching stream, max over ranks).
plain_fp64: the same batch through the FP64 engine; mixed_error: the largest
efficiency difference between the two (the accuracy bound is 1e-4).  e2e: the
mixed engine through the public C ABI (rcwa_engine_solve_batch) with host
buffers, host<->device copies inside the timed region.  --impl reference times
the CPU oracle (the NumPy restatement of the reference's LAPACK path) on the
host cores.

Multi-GPU: every rank solves its own batch of the sweep (weak scaling, no
data-path collective); only the barrier and the max of the timings cross ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RCWA solves/s on 1 B200: batched mixed vs plain FP64, max|dR,T|<=1e-4"
WORKLOAD = "2D rectangular-pillar grating Nx=Ny=10 (441 orders, 882x882), 5 patterned layers, 400x400 nm, " \
           "256 wavelengths x 8 conical angles, TE+TM"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=148, help="solve points per step per GPU (148 x 5 layers = 740 "
                    "eigensolves, five full waves on 148 SMs; the interface and tau factorisations then "
                    "fill the GPU too)")
    ap.add_argument("--nh", type=int, default=10, help="harmonics per axis (Nx=Ny)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--uneven", type=int, default=0, metavar="INSTANCES",
                    help="cfg3's uneven batch (nH 3..15, 1..10 layers, Lorentz and metal layers): the first "
                         "INSTANCES of the 4096 seeded instances as one plan, mixed and FP64")
    ap.add_argument("--surrogate", action="store_true",
                    help="the learned-surrogate pipeline (cfg4): data generation by the engine, GPU training, "
                         "tensor-core inference, surrogate plus fallback with a 2%% audit")
    ap.add_argument("--surrogate-nh", type=int, default=7,
                    help="harmonics per axis of the surrogate's training solves (cfg4: 7, i.e. 225 orders)")
    ap.add_argument("--surrogate-train", type=int, default=200000, help="training solves (cfg4: 200k)")
    ap.add_argument("--gemm-only", default=None, metavar="N,BATCH",
                    help="one batched n x n x n complex GEMM in 3xTF32 on tcgen05 and one on the FP64 path "
                         "(profiling aid)")
    ap.add_argument("--tuning", default="auto", choices=["auto", "off"],
                    help="auto: the engine's autotuner times the candidate schedules of each new (decision, "
                         "matrix order, batch class) while a plan is created, before warm-up; off: built-in rules")
    ap.add_argument("--smatrix", default=None, metavar="N,BATCH",
                    help="the z-integrator entry points: BATCH slab S-matrices and star products of order N, "
                         "end to end with host buffers")
    ap.add_argument("--conv-only", default=None, metavar="NH,POINTS",
                    help="kernel (a) alone: one plan of POINTS points of the 2D pillar sweep at NH harmonics per "
                         "axis, executed with stage timing; prints the convolution gather's time and HBM rate")
    ap.add_argument("--cfg5", type=int, default=0, metavar="POINTS",
                    help="the large-order structure: 20 circular-pillar layers (closed-form Laurent tables), "
                         "Nx=Ny=25 (2601 orders, 5202 x 5202 layer matrices), POINTS of its 32 wavelengths at "
                         "normal incidence, TE+TM, one plan execution")
    ap.add_argument("--cfg5-nh", type=int, default=25, help="harmonics per axis of --cfg5 (25: the full order)")
    ap.add_argument("--field", action="store_true",
                    help="time a field slice inside one solved point of the cfg2 stack (rcwa_plan_field)")
    ap.add_argument("--cfg5-lossless", action="store_true",
                    help="--cfg5 with lossless layers on the FP64 plan (checks |R + T - 1|)")
    ap.add_argument("--eig-only", default=None, metavar="N,BATCH",
                    help="profiling aid: one batched eigensolve of BATCH random N x N matrices, no timing line")
    return ap.parse_args()


def run_uneven(args):
    """cfg3: independent 2D-grating instances of uneven size and layer count in
    one plan (the plan bins points by harmonic grid and sizes chunks by
    memory); device time of one execution after a warm-up, for the mixed and
    the FP64 engine, and the largest efficiency difference between them."""
    import torch
    import openrcwa_b200 as o
    from openrcwa_b200 import workloads
    stacks, pts, pxy = workloads.uneven_batch(seed=0, n_instances=args.uneven)
    eng = o.Engine(0)
    stream = torch.cuda.Stream()
    res = {}
    tuner = o.Tuner() if args.tuning == "auto" else None
    runs = [("mixed", o.RCWA_PREC_MIXED, tuner), ("fp64", o.RCWA_PREC_FP64, tuner)]
    if tuner is not None and len(stacks) < 1024:
        runs.append(("mixed_untuned", o.RCWA_PREC_MIXED, None))
    tune_s = 0.0
    big = len(stacks) > 256
    for name, prec, tn in runs:
        eng.set_tuner(tn, o.RCWA_TUNING_AUTO if tn is not None else o.RCWA_TUNING_OFF)
        t0 = time.perf_counter()
        plan = eng.plan(stacks, pts, pxy, precision=prec)
        tune_s += time.perf_counter() - t0 if tn is not None else 0.0
        if big:
            # warm-up on the first 128 instances (module loading, first
            # launches), not a second pass over the whole set
            wp = eng.plan(stacks[:128], pts[:128], pxy[:128], precision=prec)
            wp.execute(stream.cuda_stream)
            stream.synchronize()
            wp.close()
        else:
            plan.execute(stream.cuda_stream)
            stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.execute(stream.cuda_stream)
        e1.record(stream)
        stream.synchronize()
        R, T, _, _, status = plan.results()
        res[name] = (e0.elapsed_time(e1), R, T, plan.launch_count(), status)
        plan.close()
    sizes = sorted({2 * s.N for s in stacks})
    # instances whose FP64 efficiencies leave [0, 1] (R + T > 1): the RTCM
    # recursion of the reference loses all accuracy there (the CPU oracle gives
    # R + T >> 1 as well), so they are counted and left out of the comparison
    R64, T64 = res["fp64"][1], res["fp64"][2]
    valid = np.all((R64 + T64 <= 1.0 + 1e-6) & (R64 >= -1e-9) & (T64 >= -1e-9), axis=1)
    valid &= (res["fp64"][4] == 0) & (res["mixed"][4] == 0)
    line = {"uneven": {"workload": ("cfg3: all 4096 seeded instances" if len(stacks) == 4096 else
                                    "cfg3 sample: first %d of the 4096 seeded instances" % len(stacks)) +
                                   ", nH 3..15 (n 98..1922), 1..10 layers, Lorentz/metal eps1, one point each, "
                                   "TE+TM, one rcwa_plan execution (one call)",
                       "instances": len(stacks), "matrix_sizes": [sizes[0], sizes[-1]],
                       "layer_eigensolves": int(sum(s.eps.shape[0] - 2 for s in stacks)),
                       "mixed_solves_per_s": len(stacks) / (res["mixed"][0] * 1e-3),
                       "fp64_solves_per_s": len(stacks) / (res["fp64"][0] * 1e-3),
                       "mixed_ms": res["mixed"][0], "fp64_ms": res["fp64"][0],
                       "unstable_instances": int(np.sum(~np.all(R64 + T64 <= 1.0 + 1e-6, axis=1))),
                       "compared_instances": int(np.sum(valid)),
                       "max_abs_dRT_mixed_vs_fp64": float(max(
                           np.max(np.abs(res["mixed"][1] - R64)[valid]),
                           np.max(np.abs(res["mixed"][2] - T64)[valid]))) if np.any(valid) else None,
                       "failed_points": {k: int(np.sum(v[4] != 0)) for k, v in res.items()},
                       "gpu_launches": res["mixed"][3]}}
    # the oracle's answers for the instances of tests/golden/uneven_sample.npz
    # that this batch contains (FP64 within 1e-9 where the oracle is
    # trustworthy, mixed within 1e-4 on the dielectric ones)
    gfile = os.path.join(ROOT, "tests", "golden", "uneven_sample.npz")
    if os.path.exists(gfile):
        g = np.load(gfile)
        d64, dmx, cnt = 0.0, 0.0, 0
        for k, i in enumerate(int(x) for x in g["ids"]):
            if i >= len(stacks) or (g["metal"][k] and not g["sane"][k]):
                continue
            cnt += 1
            d64 = max(d64, float(np.max(np.abs(R64[i] - g["R"][k]))), float(np.max(np.abs(T64[i] - g["T"][k]))))
            if not g["metal"][k]:
                dmx = max(dmx, float(np.max(np.abs(res["mixed"][1][i] - g["R"][k]))),
                          float(np.max(np.abs(res["mixed"][2][i] - g["T"][k]))))
        line["uneven"]["vs_oracle_sample"] = {"instances": cnt, "fp64_max_abs_dRT": d64, "mixed_max_abs_dRT": dmx,
                                              "fixture": "tests/golden/uneven_sample.npz"}
    if tuner is not None and "mixed_untuned" in res:
        line["uneven"]["tuning"] = {
            "mode": "auto", "plan_create_s": tune_s, "entries": len(tuner.entries()),
            "mixed_untuned_solves_per_s": len(stacks) / (res["mixed_untuned"][0] * 1e-3),
            "changed_from_builtin": [e for e in tuner.entries()
                                     if e["choice"] != tuner.default(e["op"], e["n"], 148 * e["batch_class"])]}
    print(json.dumps(line), flush=True)
    eng.close()
    return 0


def run_surrogate(args):
    """cfg4's pipeline: 200k training solves by the FP64 engine at nH
    harmonics per axis (default 7: 225 orders per solve), the network
    (4 x 256 GELU) trained on the GPU on the efficiencies of the 25 lowest
    orders (m, n in [-2, 2]) and the totals, 65,536-query batches answered by
    the network on the tensor cores and by the surrogate with fallback (hull,
    energy and 2% audit rules, fallbacks on the mixed engine), against the
    FP64 solve of the same queries."""
    import openrcwa_b200 as o
    from openrcwa_b200 import surrogate as sg
    eng = o.Engine(0)
    rng = np.random.default_rng(0)
    nh = args.surrogate_nh
    t0 = time.perf_counter()
    P = sg.sample(args.surrogate_train, rng)
    Y = sg.solve(eng, P, nh, chunk=4096)
    t_gen = time.perf_counter() - t0
    sur = sg.Surrogate(eng, nh, hidden=256, layers=4, seed=1)
    t0 = time.perf_counter()
    loss = sur.fit(P, Y, epochs=40, batch=512, lr=1e-3, seed=3)
    t_train = time.perf_counter() - t0
    Q = sg.sample(65536, rng)
    sur.predict(Q[:1024])
    t0 = time.perf_counter()
    for _ in range(5):
        Yn = sur.predict(Q)
    t_net = (time.perf_counter() - t0) / 5
    t0 = time.perf_counter()
    r = sur.query(Q, audit=0.02, seed=5)
    t_q = time.perf_counter() - t0
    t0 = time.perf_counter()
    Ys = sg.solve(eng, Q, nh, chunk=4096)
    t_solve = time.perf_counter() - t0
    t0 = time.perf_counter()
    Ym = sg.solve(eng, Q, nh, chunk=4096, precision=o.RCWA_PREC_MIXED)
    t_mixed = time.perf_counter() - t0
    err = np.abs(r["Y"] - Ys)
    net_rows = r["source"] == sg.SOURCE_NET
    line = {"surrogate": {
        "config": "cfg4%s: one-rectangle 2D grating, nH=%d harmonics per axis (%d orders) per solve, 11 parameters "
                  "-> 52 efficiencies (25 lowest orders, TE, and the totals)" % ("" if nh == 7 else " reduced", nh,
                                                                                 (2 * nh + 1) ** 2),
        "train_solves": len(P), "generation_solves_per_s": len(P) / t_gen, "train_s": t_train,
        "final_train_mse": float(loss[-1]),
        "query_batch": len(Q), "network_queries_per_s": len(Q) / t_net,
        "surrogate_with_fallback_queries_per_s": len(Q) / t_q, "fp64_solve_queries_per_s": len(Q) / t_solve,
        "mixed_solve_queries_per_s": len(Q) / t_mixed,
        "speedup_network": t_solve / t_net, "speedup_with_fallback": t_solve / t_q,
        "fallback_fraction": float(np.mean(r["source"] != sg.SOURCE_NET)),
        "fallback_by_rule": {"hull": int(np.sum(r["source"] == sg.SOURCE_HULL)),
                             "energy": int(np.sum(r["source"] == sg.SOURCE_ENERGY)),
                             "audit": int(np.sum(r["source"] == sg.SOURCE_AUDIT))},
        "fallback_precision": "mixed (3xTF32 cascade products, FP64 eigensolve)",
        "audit_max_abs_err": float(np.max(r["audit_err"])) if len(r["audit_err"]) else None,
        "rms_err_vs_solve": float(np.sqrt(np.mean(err ** 2))), "max_abs_err_vs_solve": float(np.max(err)),
        "unaudited_p99_abs_err": float(np.quantile(np.max(err[net_rows], axis=1), 0.99)) if np.any(net_rows)
        else None,
        "mixed_solve_max_abs_err_vs_fp64": float(np.max(np.abs(Ym - Ys))),
        "accuracy_target": 1e-4,
        "network_rms_err": float(np.sqrt(np.mean((Yn - Ys) ** 2)))}}
    print(json.dumps(line), flush=True)
    sur.close()
    eng.close()
    return 0


def run_gemm_only(spec):
    """Batched complex GEMMs through rcwa_zgemm_batched on seeded random
    matrices: the 3xTF32 tcgen05 kernel, then the FP64 tile kernel, for
    counter captures of those kernels; prints their relative errors."""
    import openrcwa_b200 as o
    n, b = (int(x) for x in spec.split(","))
    rng = np.random.default_rng(0)
    A = rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))
    B = rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))
    eng = o.Engine(0)
    Dm = eng.zgemm(A, B, precision=o.RCWA_PREC_MIXED)
    D6 = eng.zgemm(A, B, precision=o.RCWA_PREC_FP64)
    ref = A[0] @ B[0]
    scale = np.abs(A[0]) @ np.abs(B[0])
    print(json.dumps({"gemm_only": {"n": n, "batch": b, "tf32x3_rel_err": float(np.max(np.abs(Dm[0] - ref) / scale)),
                                    "fp64_rel_err": float(np.max(np.abs(D6[0] - ref) / scale))}}))
    eng.close()
    return 0


def run_smatrix(spec):
    """The z-integrator entry points (row a13) end to end with host buffers:
    BATCH slab S-matrices of order N (rcwa_slab_smatrix_batched) and BATCH
    star products into a running S-matrix (rcwa_star_product_batched), on
    seeded inputs: slab modes W, V near the identity, propagating and
    evanescent gamma, the uniform reference medium W0 = I.  Wall time of one
    call after a warm-up call, host copies included."""
    import openrcwa_b200 as o
    n, b = (int(x) for x in spec.split(","))
    rng = np.random.default_rng(0)

    def near_identity():
        return np.eye(n) + 0.1 * (rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))) / np.sqrt(n)

    W, V, V0 = near_identity(), near_identity(), near_identity()
    W0 = np.broadcast_to(np.eye(n, dtype=complex), (b, n, n)).copy()
    gamma = rng.uniform(0.5, 2.0, (b, n)) + 1j * rng.uniform(0.0, 0.5, (b, n))
    eng = o.Engine(0)
    out = {"n": n, "batch": b}
    for rep in range(2):
        t0 = time.perf_counter()
        Rud, Tuu, st = eng.slab_smatrix(W, V, gamma, W0, V0, 6e-7, 1e-7)
        t1 = time.perf_counter()
        S = {"Rud": np.zeros((b, n, n), complex), "Rdu": np.zeros((b, n, n), complex),
             "Tdd": np.broadcast_to(np.eye(n, dtype=complex), (b, n, n)).copy(),
             "Tuu": np.broadcast_to(np.eye(n, dtype=complex), (b, n, n)).copy()}
        S2, st2 = eng.star_product(S, {"rud": Rud, "rdu": Rud, "tdd": Tuu, "tuu": Tuu})
        t2 = time.perf_counter()
        out.update({"slab_ms": 1e3 * (t1 - t0), "slabs_per_s": b / (t1 - t0), "star_ms": 1e3 * (t2 - t1),
                    "star_products_per_s": b / (t2 - t1), "status_nonzero": int(np.sum(st != 0) + np.sum(st2 != 0)),
                    "finite": bool(np.all(np.isfinite(S2["Rud"])) and np.all(np.isfinite(S2["Tdd"]))),
                    "timing": "wall clock of one call after a warm-up call, host buffers and copies included"})
    print(json.dumps({"smatrix": out}), flush=True)
    eng.close()
    return 0 if out["status_nonzero"] == 0 and out["finite"] else 1


def conv_gather_bytes(stacks):
    """Algorithmic bytes of the convolution gather: three N x N complex128
    matrices written per distinct patterned layer (row a6 of the path)."""
    return sum(3 * 16 * s.N * s.N * (s.eps.shape[0] - 2) for s in stacks)


def run_conv_only(spec):
    """Kernel (a), the convolution-matrix gather, on the pillar workload: one
    plan of POINTS points (one stack, five patterned layers), executed three
    times with stage timing; the gather's device time of the last execution
    (CUDA events on the launching stream) and its rate against HBM."""
    import openrcwa_b200 as o
    from openrcwa_b200 import workloads
    nh, npts = (int(x) for x in spec.split(","))
    stacks, pts, pxy = workloads.pillars_2d(seed=0, nH=nh)
    eng = o.Engine(0)
    plan = eng.plan(stacks, pts[:npts], pxy[:npts])
    plan.set_profiling(True)
    for _ in range(3):
        plan.execute()
        st = plan.stage_times()
    R, T, _, _, status = plan.results()
    plan.close()
    eng.close()
    peaks, kind = measured_peaks()
    b = conv_gather_bytes(stacks)
    gbs = b / (st["conv_gather"] * 1e-3) / 1e9
    print(json.dumps({"conv_only": {"nh": nh, "points": npts, "gather_ms": st["conv_gather"],
                                    "tables_ms": st["conv_tables"], "bytes": b, "achieved_gbs": gbs,
                                    "frac_hbm": gbs / peaks["hbm_gbs"], "peak_source": kind,
                                    "status_max": int(status.max())}}))
    return 0 if status.max() == 0 else 1


def run_cfg5(args):
    """cfg5: one plan of the first POINTS wavelengths of the circular-pillar
    structure (Laurent-table layers through rcwa_plan_create_tables),
    executed once after a small warm-up plan (module loading), with stage
    timing; solves/s from the device time (CUDA events on the launching
    stream), and two size-independent checks: TE = TM (a centred disk is C4
    symmetric and the incidence is normal) and 0 <= R, T, R + T <= 1.  With
    --cfg5-lossless the layers are lossless and the plan FP64: |R + T - 1| is
    then the check.  The roofline is the Schur stage (nominal 81.33 n^3 flops
    per matrix) against the DGEMM rate measured in the same run."""
    import torch
    import openrcwa_b200 as o
    from openrcwa_b200 import workloads
    nh, npts = args.cfg5_nh, args.cfg5
    lossless = args.cfg5_lossless
    prec = o.RCWA_PREC_FP64 if lossless else o.RCWA_PREC_MIXED
    stacks, pts, pxy = workloads.circular_pillars(seed=0, nH=nh, lossless=lossless)
    eng = o.Engine(0)
    stream = torch.cuda.Stream()
    ws, wp, wx = workloads.circular_pillars(seed=0, nH=3, n_lambda=2, n_layers=3)
    w = eng.plan(ws, wp, wx, precision=prec)
    w.execute(stream.cuda_stream)
    stream.synchronize()
    w.close()
    fp64_peak = fp64_gemm_peak_tflops(torch)
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    plan = eng.plan(stacks, pts[:npts], pxy[:npts], precision=prec)
    t_create = time.perf_counter() - t0
    plan.set_profiling(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(0)
    clocks.start()
    e0.record(stream)
    plan.execute(stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    stages = plan.stage_times()
    R, T, _, _, status = plan.results()
    chunks = plan.schedule()
    plan.close()
    eng.close()
    n = 2 * stacks[0].N
    nj = int(npts * (stacks[0].thickness.size - 2))
    schur_flops = 81.33 * float(n) ** 3 * nj
    out = {
        "workload": "20 circular-pillar layers (closed-form disk Laurent tables, radius/period U(0.2, 0.45), "
                    "thickness U(20, 100) nm, eps1 alternating 4.0 / %s, eps2 1), substrate 2.25, period "
                    "400 nm, Nx=Ny=%d (%d orders, %d x %d layer matrices), first %d of 32 wavelengths 500-900 nm, "
                    "normal incidence, TE+TM" % ("2.1" if lossless else "2.1+0.01i", nh, stacks[0].N, n, n, npts),
        "precision": ("fp64" if lossless else
                      "mixed: cascade products, modal V and blocked-LU updates 3xTF32 on tcgen05, "
                      "eigensolve FP64"),
        "solves_per_s": npts / (ms * 1e-3), "ms_per_execution": ms, "plan_create_s": t_create,
        "chunks": len(chunks), "eigensolves": nj,
        "ctas_per_matrix": {"eigensolver": o.eig_cluster_size(n, nj // max(1, len(chunks))),
                            "lu_panel_interfaces": o.lu_cluster_size(n, 2),
                            "lu_panel_tau": o.lu_cluster_size(n, 1)},
        "stage_ms": {k: round(v, 1) for k, v in stages.items() if v > 1.0},
        "roofline": {"kernel": "schur_qr", "bound": "tensor", "achieved": schur_flops / (stages["schur_qr"] * 1e9),
                     "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": schur_flops / (stages["schur_qr"] * 1e9) / fp64_peak,
                     "peak_source": "FP64 DGEMM measured in this run (cuBLAS via torch)",
                     "note": "nominal 81.33 n^3 flops per matrix (LAPACK's count for the standard QR iteration)"},
        "status_max": int(status.max()),
        "max_abs_TE_minus_TM": float(np.max(np.abs(R[:, 0] - R[:, 1]))),
        "R_range": [float(R.min()), float(R.max())], "R_plus_T_max": float(np.max(R + T)),
        "clocks": clk}
    if lossless:
        out["max_abs_R_plus_T_minus_1"] = float(np.max(np.abs(R + T - 1.0)))
    print(json.dumps({"cfg5": out}), flush=True)
    return 0 if status.max() == 0 else 1


def run_field(args):
    """Field slices inside one solved point of the cfg2 stack (rcwa_plan_field:
    the intermediate mode amplitudes and saveFieldImage's XZ slice of Ex at
    500 columns), timed end to end per call (the call synchronises), beside
    the oracle's restatement of the same slice on the host cores."""
    import openrcwa_b200 as o
    import oracle.rcwa_oracle as orc
    from openrcwa_b200 import workloads
    nh = args.nh
    stacks, pts, pxy = workloads.pillars_2d(seed=0, nH=nh)
    eng = o.Engine(0)
    plan = eng.plan(stacks, pts[:1], pxy[:1])
    plan.execute()
    px, py = pxy[0, 0]
    f = plan.field(0, px, py, 1, 0.0, 0, nres1=500)  # warm-up (module loading, allocations)
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        f = plan.field(0, px, py, 1, 0.0, 0, nres1=500)
    t_gpu = (time.perf_counter() - t0) / reps
    plan.close()
    eng.close()
    st = stacks[0]
    s = orc.RCWASolver(st.nHx, st.nHy)
    for l in range(st.eps.shape[0]):
        s.addLayer(orc.OracleLayer(st.cx, st.cy, st.eps[l]))
    s.setBlochWavevector(pts[0, 2], pts[0, 3])
    t0 = time.perf_counter()
    s.solve(pts[0, 1], list(range(st.eps.shape[0])), list(st.thickness))
    c = s.generateHorizontalPlaneWave(px, py, 0)
    t_solve = time.perf_counter() - t0
    inp = [(i, v) for i, v in enumerate(c) if abs(v) > 1e-14]
    t0 = time.perf_counter()
    fo = s.fieldSlice(1, 0.0, 0, inp, list(range(st.eps.shape[0])), list(st.thickness), nRes1=500)
    t_cpu = time.perf_counter() - t0
    print(json.dumps({"field": {
        "workload": "XZ slice of Ex (500 x %d samples) inside one point of the cfg2 stack (Nx=Ny=%d, n = %d, "
                    "5 interior layers)" % (f.shape[0], nh, 2 * st.N),
        "gpu_s_per_slice": t_gpu, "cpu_oracle_s_per_slice": t_cpu, "cpu_oracle_solve_s": t_solve,
        "max_abs_vs_oracle": float(np.max(np.abs(f - fo))), "max_abs_field": float(np.max(np.abs(fo)))}}),
          flush=True)
    return 0


def run_eig_only(spec):
    """One rcwa_zgeev_batched call on seeded random matrices (the kernels of the
    per-layer eigenproblem alone), for counter captures of those kernels."""
    import openrcwa_b200 as o
    n, b = (int(x) for x in spec.split(","))
    rng = np.random.default_rng(0)
    A = rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))
    eng = o.Engine(0)
    w, V, info = eng.zgeev(A)
    res = np.abs(A[0] @ V[0] - V[0] * w[0][None, :]).max() / np.abs(A[0]).max()
    print(json.dumps({"eig_only": {"n": n, "batch": b, "info_max": int(info.max()), "residual": float(res)}}))
    eng.close()
    return 0 if info.max() == 0 else 1


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp64_gemm_peak_tflops(torch):
    """cuBLAS DGEMM throughput (torch.matmul float64, 8192^3, best of 5): the
    FP64 denominator of the eigensolver roofline (the pool's peak file has
    only HBM and BF16)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def tf32_gemm_peak_tflops(torch):
    """cuBLAS TF32 GEMM throughput (torch.matmul float32 with TF32 allowed,
    8192^3, best of 5): the denominator of the 3xTF32 tensor-core products."""
    n = 8192
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(n, n, dtype=torch.float32, device="cuda")
    b = torch.randn(n, n, dtype=torch.float32, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return best


def eig_flops(n):
    """Algorithmic real flops of one complex eigen-decomposition with
    eigenvectors, split as in Golub & Van Loan (complex = 4x real counts):
    Hessenberg + Q accumulation 4.67 n^3 x 4, QR iteration with T and Z
    20.33 n^3 x 4 (together 25 n^3 x 4 = 100 n^3)."""
    return {"hessenberg": 18.67 * n ** 3, "schur_qr": 81.33 * n ** 3, "total": 100.0 * n ** 3}


def cpu_solve_sample(stacks, pts, pxy, count, threads=None):
    """Time `count` solves of the oracle on the host (all BLAS threads, or
    `threads`).  Returns (seconds, per point: (R, T, REF, TRN) of its
    polarisations)."""
    import oracle.rcwa_oracle as orc
    from threadpoolctl import threadpool_limits
    st = stacks[0]
    out = []
    with threadpool_limits(limits=threads):
        t0 = time.perf_counter()
        for p in range(count):
            _, lam, kx0, ky0 = pts[p]
            s = orc.RCWASolver(st.nHx, st.nHy)
            for l in range(st.eps.shape[0]):
                s.addLayer(orc.OracleLayer(st.cx, st.cy, st.eps[l]))
            s.setBlochWavevector(kx0, ky0)
            s.solve(lam, list(range(st.eps.shape[0])), list(st.thickness))
            k0 = 2 * np.pi / lam
            r = []
            for e in range(pxy.shape[1]):
                c = s.generateHorizontalPlaneWave(pxy[p, e, 0], pxy[p, e, 1], 0)
                r.append(s.scatterPlaneWave(c, 0, st.eps.shape[0] - 1, k0))
            out.append((np.array([a.sum() for a, _ in r]), np.array([b.sum() for _, b in r]),
                        np.array([a for a, _ in r]), np.array([b for _, b in r])))
        return time.perf_counter() - t0, out


def run_reference(args):
    from openrcwa_b200 import workloads
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    stacks, pts, pxy = workloads.pillars_2d(seed=0, nH=args.nh)
    for _ in range(args.warmup):
        cpu_solve_sample(stacks, pts, pxy, 1)
    tt = 0.0
    for k in range(args.steps):
        tt += cpu_solve_sample(stacks, pts[k:], pxy[k:], 1)[0]
    value = args.steps / tt
    cores = os.cpu_count()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": "1 solve per step", "parallelism": "host BLAS threads"},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} solves of the sweep (points 0..{args.steps - 1}), "
                                       "NumPy/OpenBLAS zgeev path, all host threads"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.eig_only:
        return run_eig_only(args.eig_only)
    if args.conv_only:
        return run_conv_only(args.conv_only)
    if args.cfg5:
        return run_cfg5(args)
    if args.field:
        return run_field(args)
    if args.gemm_only:
        return run_gemm_only(args.gemm_only)
    if args.smatrix:
        return run_smatrix(args.smatrix)
    if args.surrogate:
        return run_surrogate(args)
    if args.uneven:
        return run_uneven(args)
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist

    import openrcwa_b200 as o
    from openrcwa_b200 import workloads

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def allmax(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    stacks, pts, pxy = workloads.pillars_2d(seed=0, nH=args.nh)
    N = stacks[0].N
    n = 2 * N
    B = args.batch
    eng = o.Engine(local)
    tuner = None
    if args.tuning == "auto":
        tuner = o.Tuner()
        eng.set_tuner(tuner, o.RCWA_TUNING_AUTO)
    plan_info = {}
    bpts, bpxy = workloads.batch_slice(pts, pxy, workloads.shard_start(rank, world, B, 0), B)
    stream = torch.cuda.Stream()
    fp64_peak = fp64_gemm_peak_tflops(torch)
    tf32_peak = tf32_gemm_peak_tflops(torch)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed_plan(precision, warmup, sample_clocks):
        """Warm up, then time `steps` executions of one plan of this rank's
        batch on `stream` (CUDA events, max over ranks).  Stage-timing events
        are on from the start: the second execution captures the launch
        sequence (with its event records) into the CUDA graph that every later
        execution launches.  The stage times of each execution are read
        before the next one starts (a host wait on the last stage event
        inside the timed region): consecutive graph launches therefore do not
        overlap, which leaves the measured rate slightly pessimistic."""
        tc0 = time.perf_counter()
        plan = eng.plan(stacks, bpts, bpxy, precision=precision)
        plan_info[precision] = {"plan_create_s": time.perf_counter() - tc0, "schedule": plan.schedule()}
        plan.set_profiling(True)
        for _ in range(warmup):
            plan.execute(stream.cuda_stream)
        stream.synchronize()
        barrier()
        clocks = ClockSampler(local) if sample_clocks else None
        if clocks:
            clocks.start()
        stage_ms = {}
        e0.record(stream)
        for _ in range(args.steps):
            plan.execute(stream.cuda_stream)
            for k, v in plan.stage_times().items():
                stage_ms[k] = stage_ms.get(k, 0.0) + v
        e1.record(stream)
        stream.synchronize()
        clk = clocks.stop() if clocks else None
        t_ms = allmax(e0.elapsed_time(e1))
        launches = plan.launch_count() * args.steps
        R, T, REF, TRN, status = plan.results(orders=True)
        if np.any(status):
            raise SystemExit(f"solve status {status}")
        # release the plan (and with it the engine's cached workspace) so that
        # the next plan and the end-to-end calls find the workspace free
        plan.close()
        return t_ms, stage_ms, launches, clk, (R, T, REF, TRN)

    # the headline: the mixed-precision engine; then the plain FP64 engine on
    # the same batch, whose results (parity-tested against the oracle at 1e-9)
    # measure the mixed path's error
    t_ms, stage_ms, launches, clk, res_mixed = timed_plan(o.RCWA_PREC_MIXED, args.warmup, True)
    t64_ms, stage64_ms, _, _, res_fp64 = timed_plan(o.RCWA_PREC_FP64, max(2, min(args.warmup, 3)), False)
    value = world * B * args.steps / (t_ms * 1e-3)
    value64 = world * B * args.steps / (t64_ms * 1e-3)
    dRT = max(float(np.max(np.abs(res_mixed[0] - res_fp64[0]))), float(np.max(np.abs(res_mixed[1] - res_fp64[1]))))
    dorders = max(float(np.max(np.abs(res_mixed[2] - res_fp64[2]))), float(np.max(np.abs(res_mixed[3] - res_fp64[3]))))

    # e2e: the public C ABI with host buffers, a different batch each step
    barrier()
    h2d = d2h = 0
    t0 = time.perf_counter()
    for k in range(args.steps):
        p2, x2 = workloads.batch_slice(pts, pxy, workloads.shard_start(rank, world, B, k + 1), B)
        R2, T2, _, _, st2 = eng.solve_batch(stacks, p2, x2, orders=False, precision=o.RCWA_PREC_MIXED)
        st = stacks[0]
        h2d += st.eps.nbytes + st.cx.nbytes + st.cy.nbytes + st.thickness.nbytes + p2.nbytes + x2.nbytes
        d2h += R2.nbytes + T2.nbytes + st2.nbytes
    barrier()
    e2e_s = allmax(time.perf_counter() - t0)
    e2e = world * B * args.steps / e2e_s

    # the 1D lamellar grating (11 orders, 16 frequencies): one plan replayed
    # as a CUDA graph, and the same solve through the C ABI with host buffers
    g_st, g_pts, g_pxy = workloads.grating_1d(16, 5)
    gplan = eng.plan(g_st, g_pts, g_pxy)
    for _ in range(3):
        gplan.execute(stream.cuda_stream)
    reps = 50
    barrier()
    e0.record(stream)
    for _ in range(reps):
        gplan.execute(stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    g_ms = allmax(e0.elapsed_time(e1))
    g_launch = gplan.launch_count()
    gplan.close()
    for _ in range(10):   # untimed warm-up calls of the end-to-end path
        eng.solve_batch(g_st, g_pts, g_pxy, orders=True)
    barrier()
    t0 = time.perf_counter()
    for _ in range(reps):
        eng.solve_batch(g_st, g_pts, g_pxy, orders=True)
    g_e2e_s = allmax(time.perf_counter() - t0)
    grating = {"workload": "1D lamellar grating Nx=5 (11 orders, 22x22), 16 frequencies, TE+TM",
               "value": len(g_pts) * reps / (g_ms * 1e-3), "e2e": len(g_pts) * reps / g_e2e_s,
               "unit": "solves/s", "ms_per_sweep": g_ms / reps, "gpu_launches_per_sweep": g_launch,
               "graph": "plan replayed as one CUDA graph per sweep"}

    # roofline of the dominant stage
    peaks, peak_kind = measured_peaks()
    per_launch = {k: v / args.steps for k, v in stage_ms.items()}
    dom = max(per_launch, key=per_launch.get)
    jobs = B * (stacks[0].eps.shape[0] - 2)
    fl = eig_flops(n)
    roof = None
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            per_matrix = json.load(f).get(dom + "_per_matrix")
        traffic = per_matrix * jobs if per_matrix else None
    if dom in ("schur_qr", "hessenberg"):
        achieved = fl[dom] * jobs / (per_launch[dom] * 1e-3) / 1e12
        roof = {"kernel": dom, "bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "traffic": traffic,
                "peak_source": "FP64 DGEMM measured in this run (cuBLAS via torch)",
                "flops_per_launch": fl[dom] * jobs, "ms_per_launch": per_launch[dom]}
    # the tensor-core products of the cascade: 4 complex GEMMs of n^3 per
    # interface step, each 3 TF32 products (hi*hi, hi*lo, lo*hi) of 8 n^3 flops
    n_iface = stacks[0].eps.shape[0] - 1
    tc_ms = per_launch.get("cascade_gemm", 0.0)
    tc_flops = 3 * 4 * 8.0 * n ** 3 * n_iface * B
    tensor_gemm = None
    if tc_ms > 0:
        ach = tc_flops / (tc_ms * 1e-3) / 1e12
        tensor_gemm = {"kernel": "zgemm_tf32x3 (tcgen05 kind::tf32)", "bound": "tensor", "achieved": ach,
                       "peak": tf32_peak, "unit": "TFLOP/s", "frac": ach / tf32_peak if tf32_peak else None,
                       "peak_source": "cuBLAS TF32 GEMM measured in this run (torch.matmul float32, TF32 on)",
                       "flops_per_step": tc_flops, "ms_per_step": tc_ms}
    conv_ms = per_launch.get("conv_gather", 0.0)
    conv_roof = None
    if conv_ms > 0:
        cb = conv_gather_bytes(stacks)
        ach = cb / (conv_ms * 1e-3) / 1e9
        conv_roof = {"kernel": "conv_gather_kernel (row a6, block-Toeplitz gather)", "bound": "hbm",
                     "achieved": ach, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": ach / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None,
                     "bytes_per_launch": cb, "ms_per_launch": conv_ms,
                     "note": "three N x N complex128 matrices written per distinct patterned layer; the sweep "
                             "shares one stack, so one launch per step"}
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128 with tf32x3 cascade products", "data": "synthetic",
            "config": {"workload": WORKLOAD, "batch_points_per_gpu": B, "orders": N, "matrix": n,
                       "precision": "mixed: cascade GEMMs, modal V products and the K = 128 updates of the "
                                    "blocked interface/tau LU factorisations and solves 3xTF32 on tcgen05 (FP32 "
                                    "accumulation within K-blocks, FP64 across); eigensolve, LU panels and "
                                    "triangles, half-spaces and efficiency sums FP64",
                       "parallelism": f"replicas x{world}",
                       "l2": "per-step working set several GB > 126 MB L2"},
            "outputs_per_s": {"value": value * bpxy.shape[1], "unit": "(point, polarisation) R/T outputs/s",
                              "note": "each solve serves both polarisations from one S-matrix"},
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps},
            "gpu_launches": launches, "clocks": clk, "roofline": roof, "tensor_gemm": tensor_gemm,
            "conv_gather": conv_roof,
            "plain_fp64": {"value": value64, "unit": "solves/s", "ms_per_step": t64_ms / args.steps,
                           "stage_ms_per_step": {k: v / args.steps for k, v in stage64_ms.items()}},
            "mixed_error": {"max_abs_dRT_vs_fp64": dRT, "max_abs_dorder_vs_fp64": dorders, "bound": 1e-4,
                            "reference": "the FP64 engine on the same batch (1e-9 of the oracle in the tests)"},
            "grating_1d": grating,
            "schedule": plan_info[o.RCWA_PREC_MIXED]["schedule"],
            "tuning": {"mode": args.tuning,
                       "plan_create_s": plan_info[o.RCWA_PREC_MIXED]["plan_create_s"],
                       "entries": tuner.entries() if tuner is not None else []},
            "stage_ms_per_step": per_launch, "peaks": {"fp64_dgemm_tflops": fp64_peak, "tf32_gemm_tflops": tf32_peak,
                                                       "hbm_gbs": peaks.get("hbm_gbs"), "source": peak_kind}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the oracle on points 0 and 1 of the timed batch: the CPU baseline
        # (all host threads, then one thread as in the reference's serial
        # frequency loop), and the error of both engines against it
        tcpu, ref_pts = cpu_solve_sample(stacks, bpts, bpxy, 1)
        t1, ref1 = cpu_solve_sample(stacks, bpts[1:], bpxy[1:], 1, threads=1)
        line["cpu_baseline"] = {"value": 1.0 / tcpu, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": "1 solve (point 0 of the timed batch) through the NumPy oracle "
                                          "(LAPACK zgeev path), all host BLAS threads",
                                "single_thread": {"value": 1.0 / t1, "unit": "solves/s", "cores": 1,
                                                  "sample": "point 1 of the timed batch, one BLAS thread"}}
        N_ = stacks[0].N
        errs = {"mixed": 0.0, "fp64": 0.0}
        for k, (Ro, To, REFo, TRNo) in ((0, ref_pts[0]), (1, ref1[0])):
            for name, res in (("mixed", res_mixed), ("fp64", res_fp64)):
                R_, T_, REF_, TRN_ = res
                ords = np.abs(REF_.reshape(B, -1, N_)[k] - REFo).max(), np.abs(TRN_.reshape(B, -1, N_)[k] - TRNo).max()
                errs[name] = max(errs[name], float(np.abs(R_[k] - Ro).max()), float(np.abs(T_[k] - To).max()),
                                 float(max(ords)))
        line["mixed_error"]["max_abs_vs_oracle"] = errs["mixed"]
        line["mixed_error"]["fp64_max_abs_vs_oracle"] = errs["fp64"]
        line["mixed_error"]["oracle_points"] = "points 0 and 1 of the timed batch, every R, T and per-order value"
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
