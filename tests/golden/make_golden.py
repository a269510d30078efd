"""Generates the golden fixtures under tests/golden/ from the reference tree.

Run once in a container that has the reference checkout:
    python tests/golden/make_golden.py [/root/reference]

Outputs (committed; nothing at test time reads the reference tree):
  inp/<dir>__<name>.inp       the sample input files (sample_input/**.inp)
  quick_test.json             statistics of the shipped quick_test run
                              (sample_input/quick_test/executed_job)
  quick_test_events.npz       the first 2000 per-event FPT / FPT2 / TPT / TPT2
                              times of every lane (in steps), decoded from
                              the four .restart files of that run
  quick_test_rank{0..3}.restart.xz
                              the .restart files of ranks 0-3 of that run,
                              as the reference wrote them (xz-compressed):
                              the fixtures of the restart reader and writer
  quick_test_outputs/         that run's output files (.log, .dat) and one
                              of its WRITEX trajectory dumps (.log.xz), as
                              the reference wrote them

The .restart layout decoded here is the reference's
LangevinEquationSIMDMultiple::WriteRestartFile (src/langevinDynamicsSingleBarrier.h:1048-1136)
followed by TrajectoryData::WriteRestartFile (S.h:385-576), the barrier
table (src/DataLocator.h:167-174) and the overdamped random force
(S.h:2776-2785): little-endian int32 / uint64 / float64.
"""
import glob
import json
import os
import shutil
import struct
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
OUT = os.path.dirname(os.path.abspath(__file__))


def copy_inputs():
    os.makedirs(os.path.join(OUT, "inp"), exist_ok=True)
    for f in sorted(glob.glob(os.path.join(REF, "sample_input", "*", "*.inp"))):
        d = os.path.basename(os.path.dirname(f))
        shutil.copy(f, os.path.join(OUT, "inp", f"{d}__{os.path.basename(f)}"))


def read_log_stats(path):
    """'# average / # sd / # count' triples, in file order."""
    out = []
    cur = {}
    for line in open(path):
        w = line.split()
        if len(w) >= 3 and w[0] == "#" and w[1] in ("average", "sd", "count"):
            cur[w[1]] = float(w[2]) if w[1] != "count" else int(w[2])
            if w[1] == "count":
                out.append(cur)
                cur = {}
    return out


def read_hist(path):
    rows = []
    meta = {}
    for line in open(path):
        w = line.split()
        if not w:
            continue
        if w[0] == "#" and len(w) == 3 and w[1] in ("HMin", "HMax", "HBin", "NBin"):
            meta[w[1]] = float(w[2])
        elif w[0] == "#" and len(w) >= 4 and w[1] in ("R", "Nwt"):
            meta[w[1]] = float(w[3])
        elif w[0] != "#":
            rows.append([float(x) for x in w])
    return meta, rows


def read_dat(path):
    return list(np.fromfile(path, dtype="<f8"))


class Reader:
    def __init__(self, b):
        self.b = b
        self.o = 0

    def i32(self):
        v = struct.unpack_from("<i", self.b, self.o)[0]
        self.o += 4
        return v

    def u64(self):
        v = struct.unpack_from("<Q", self.b, self.o)[0]
        self.o += 8
        return v

    def f64(self):
        v = struct.unpack_from("<d", self.b, self.o)[0]
        self.o += 8
        return v

    def vec(self):
        n = self.u64()
        a = np.frombuffer(self.b, dtype="<f8", count=n, offset=self.o).copy()
        self.o += 8 * n
        return a

    def ivec(self, n):
        a = np.frombuffer(self.b, dtype="<i4", count=n, offset=self.o).copy()
        self.o += 4 * n
        return a


def decode_restart(path):
    r = Reader(open(path, "rb").read())
    sig = r.i32()
    assert sig == 2345, sig
    W = r.i32()
    hdr = {"W": W}
    hdr["x0"], hdr["v0"], hdr["gamma"], hdr["kb"], hdr["T"], hdr["m"] = [r.f64() for _ in range(6)]
    hdr["dt"] = r.f64()
    hdr["nsteps"] = r.u64()
    hdr["wt"] = r.i32()
    hdr["freq_stat"] = r.u64()
    hdr["freq_save"] = r.u64()
    _save = [r.i32() for _ in range(4)]
    _rand = [r.i32() for _ in range(2)]
    hdr["L"], hdr["H0"], hdr["H1"], hdr["init_state"] = [r.f64() for _ in range(4)]
    _ = [r.i32() for _ in range(2)]
    hdr["q"], hdr["tau"], hdr["eta0"] = [r.f64() for _ in range(3)]
    _ = [r.i32() for _ in range(3)]
    hdr["rank"] = r.i32()
    hdr["rng"] = [(r.u64(), r.u64()) for _ in range(3)]
    assert r.i32() == 9998
    wt = r.i32()
    fpt = r.i32()
    lanes = []
    for _lane in range(W):
        L = {}
        L["x"], L["v"], L["f"], L["e"], L["eta"], L["barrier"] = [r.f64() for _ in range(6)]
        series = [r.vec() for _ in range(8)]
        L["traj_x"] = series[0]
        L["state"], _prev, _sp, _sn, _h = [r.f64() for _ in range(5)]
        L["state_count"] = [r.f64(), r.f64()]
        _idx = [r.f64() for _ in range(4)]
        _ = [r.i32() for _ in range(2)]
        L["v0"], _eta0, L["state0"] = [r.f64() for _ in range(3)]
        _ = [r.f64() for _ in range(4)]
        _ = [r.i32() for _ in range(2)]
        if wt:
            _tick_prev = r.f64()
            _passed = r.i32()
            L["ticks"] = r.vec()
        if fpt:
            L["fpt"] = r.vec()
            L["instant"] = r.vec()
            L["initial"] = r.vec()
            _ = r.f64(); _ = r.i32(); _ = r.f64(); _ = r.f64(); _ = r.i32(); _ = r.i32()
            L["fpt2"] = r.vec()
            _ = r.f64(); _ = r.i32(); _ = r.i32(); _ = r.i32()
        # TPT and CG blocks are present in the quick_test run (TPT true, FPTCG true)
        L["tpt"] = r.vec()
        _ = r.f64(); _ = r.i32()
        L["tpt2"] = r.vec()
        _ = r.f64(); _ = r.i32(); _ = r.i32()
        ncg = r.u64()
        sizes = r.ivec(ncg)
        L["cg"] = {}
        for j in range(ncg):
            L["cg"][int(sizes[j])] = r.vec()
            _ = r.f64(); _ = r.i32(); _ = r.i32()
        lanes.append(L)
    ncell = r.u64()
    for _ in range(ncell):
        for _l in range(W):
            r.i32()
            r.u64()
    _min_id = r.i32()
    _rf = [r.f64() for _ in range(W)]
    assert r.i32() == 9990
    assert r.o == len(r.b)
    return hdr, lanes


def main():
    copy_inputs()
    ej = os.path.join(REF, "sample_input", "quick_test", "executed_job")
    base = os.path.join(ej, "m1.0_t1.00e-05_0")
    g = {}
    for name in ("firstPassageTime", "firstPassageTime2", "transitionPathTime", "transitionPathTime2"):
        g[name] = read_log_stats(base + f"_{name}.log")[0]
        g[name]["per_traj"] = read_dat(base + f"_{name}.dat")
    cg = read_log_stats(base + "_firstPassageTimeCG2.log")
    sizes = [2, 3, 4, 5, 10, 100, 1000]
    g["firstPassageTimeCG2"] = []
    for j, s in enumerate(sizes):
        e = dict(cg[j])
        e["size"] = s
        e["per_traj"] = read_dat(base + f"_firstPassageTimeCG2_{j:04d}_{s:04d}.dat")
        g["firstPassageTimeCG2"].append(e)
    sc = []
    for line in open(base + "_stateCount.log"):
        w = line.split()
        if len(w) >= 5 and w[1] == "state":
            sc.append(int(w[3]))
    g["stateCount"] = sc
    msd = [[float(x) for x in line.split()] for line in open(base + "_msd.log") if not line.startswith("#")]
    g["msd"] = msd
    meta, rows = read_hist(base + "_waitingTime.log")
    g["waitingTime"] = {"meta": meta, "counts": [r[3] for r in rows], "percent": [r[4] for r in rows]}
    meta, rows = read_hist(base + "_State0Distribution.log")
    g["State0Distribution"] = {"meta": meta, "counts": [r[3] for r in rows]}
    for name in ("initialBarrierHeightHistogram", "instantBarrierHeightHistogram"):
        meta, rows = read_hist(base + f"_{name}.log")
        g[name] = {"meta": meta, "nonzero": [[i, r[3], r[4]] for i, r in enumerate(rows) if r[3] != 0]}
    # The PrintParameter header block, for output-format tests.
    hdr = []
    for line in open(base + "_firstPassageTime.log"):
        if line.startswith("# average"):
            break
        hdr.append(line.rstrip("\n"))
    g["print_parameter_header"] = hdr
    g["time_log"] = open(base + "_time.log").read().splitlines()
    with open(os.path.join(OUT, "quick_test.json"), "w") as f:
        json.dump(g, f, indent=1)

    keep = 2000   # events kept per lane and list (first ones, in event order)
    ev = {k: [] for k in ("fpt", "fpt2", "tpt", "tpt2")}
    lane_means = []
    lane_counts = []
    for rank in range(4):
        hdr, lanes = decode_restart(os.path.join(ej, f"m1.0_t1.00e-05_restart_0_{rank:05d}_00000.restart"))
        dt = hdr["dt"]
        for L in lanes:
            for k in ("fpt", "fpt2", "tpt", "tpt2"):
                ev[k].append(np.rint(L[k][:keep] / dt).astype(np.int64))
            lane_means.append(float(np.mean(L["fpt"])))
            lane_counts.append(len(L["fpt"]))
    np.savez_compressed(
        os.path.join(OUT, "quick_test_events.npz"),
        **{k: np.concatenate(v).astype(np.int32) for k, v in ev.items()},
        lane_counts=np.array(lane_counts),
        lane_fpt_means=np.array(lane_means),
    )
    print("fpt lanes", lane_counts)
    import lzma
    for rank in range(4):
        src = os.path.join(ej, f"m1.0_t1.00e-05_restart_0_{rank:05d}_00000.restart")
        dst = os.path.join(OUT, f"quick_test_rank{rank}.restart.xz")
        with open(src, "rb") as f, lzma.open(dst, "wb", preset=9) as g:
            g.write(f.read())
    outs = os.path.join(OUT, "quick_test_outputs")
    os.makedirs(outs, exist_ok=True)
    for name in sorted(os.listdir(ej)):
        if name.startswith("m1.0_t1.00e-05_0_") and "trajectory" not in name:
            shutil.copyfile(os.path.join(ej, name), os.path.join(outs, name))
    # one WRITEX trajectory dump (trial 0, lane 1, rank 2), xz-compressed
    name = "m1.0_t1.00e-05_0_trajectory_0000000000_0000000001_0000000002.log"
    with open(os.path.join(ej, name), "rb") as f, lzma.open(os.path.join(outs, name + ".xz"), "wb", preset=9) as g:
        g.write(f.read())


if __name__ == "__main__":
    main()
