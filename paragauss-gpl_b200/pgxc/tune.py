"""Autotuner for the XC build's batching parameters.

The reference has one knob for this: machineparameters_veclen (vla), the
number of grid points a batch holds (modules/machineparameters_module.f90:67,
range 1..10000 at :152-155), handed out by more_grid in contiguous slices
(modules/grid_module.f90:1133-1181).  Here the point batch is fixed by the
tensor-core tile (128 points: the MMA M of the INT8 contractions), and what
decides the throughput is how many tiles go into one launch of the
persistent kernels:

  max_chunk_points  points (whole 128-point tiles) processed per chunk:
                    one launch of each kernel per chunk.  Larger chunks
                    amortise launch and pipeline fill over more tiles and
                    keep all 148 SMs busy; smaller ones keep the per-chunk
                    basis values (32 B per slot and point) small.

A tuning run times the build of representative workloads for every
candidate and writes a table keyed by workload class; the library's
callers look the class of their workload up (choose) and pass the result
in pgxc_options.  The committed table (tune_b200.json, beside this file)
was measured on one B200; classes not in it fall back to the defaults
(chunks sized from free device memory).

Workload classes: "single" builds by the precision and by buckets of basis
size and grid size; "set" builds (many molecules through pgxc_batch, one
launch per kernel over all their tiles) by total grid size.
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tune_b200.json")

# bucket edges (upper bounds, inclusive); the last bucket is open
NBAS_EDGES = (64, 256, 1024, 4096)
NPTS_EDGES = (65536, 1 << 20, 1 << 23)
CANDIDATES = (65536, 262144, 1 << 20, 0)   # max_chunk_points; 0: sized from free device memory


def bucket(x, edges):
    for i, e in enumerate(edges):
        if x <= e:
            return i
    return len(edges)


def single_key(nbas, npts, precision):
    return f"single:{precision}:nbas{bucket(nbas, NBAS_EDGES)}:npts{bucket(npts, NPTS_EDGES)}"


def set_key(total_pts):
    return f"set:mixed:npts{bucket(total_pts, NPTS_EDGES)}"


def load(path=TABLE):
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f).get("entries", {})


def choose(key, table=None):
    """max_chunk_points for a workload class (0: the library's default)."""
    t = load() if table is None else table
    e = t.get(key)
    return int(e["max_chunk_points"]) if e else 0


def choose_single(case, precision, table=None):
    return choose(single_key(case.nbas, case.npts, precision), table)


def choose_set(cases_, table=None):
    return choose(set_key(sum(c.npts for c in cases_)), table)


def best(timings):
    """The candidate with the smallest time; ties go to the larger chunk."""
    ok = {k: v for k, v in timings.items() if v is not None}
    if not ok:
        return None
    return min(ok, key=lambda k: (ok[k], -(k if k > 0 else 1 << 62)))


def tune_single(case, precision, time_build, candidates=CANDIDATES):
    """time_build(case, precision, max_chunk_points) -> ms (None: not possible)."""
    t = {c: time_build(case, precision, c) for c in candidates}
    return single_key(case.nbas, case.npts, precision), t, best(t)


def tune_set(cases_, time_set, candidates=CANDIDATES):
    """time_set(cases, max_chunk_points) -> ms per set (None: not possible)."""
    t = {c: time_set(cases_, c) for c in candidates}
    return set_key(sum(c.npts for c in cases_)), t, best(t)


def write(entries, path=TABLE, device=""):
    with open(path, "w") as f:
        json.dump({"device": device, "candidates": list(CANDIDATES), "nbas_edges": list(NBAS_EDGES),
                   "npts_edges": list(NPTS_EDGES), "entries": entries}, f, indent=1, sort_keys=True)


def _run(argv=None):
    """Measure on the current GPU and write the table (python -m pgxc.tune)."""
    import argparse
    import torch
    from . import cases, lib

    p = argparse.ArgumentParser()
    p.add_argument("--out", default=TABLE)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--set-size", type=int, default=256)
    args = p.parse_args(argv)

    def timer(fn, steps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def time_build(case, precision, chunk):
        try:
            ctx = lib.Context(case, precision=precision, weighted=False, max_chunk_points=chunk,
                              screen_threshold=1e-10)
        except lib.PgxcError:
            return None
        dC = torch.from_numpy(case.c_fortran()).cuda()
        docc = torch.from_numpy(case.occ_fortran()).cuda()
        dham = torch.zeros(case.xc_length, dtype=torch.float64, device="cuda")
        dsum = torch.zeros(2, dtype=torch.float64, device="cuda")
        try:
            return timer(lambda: ctx.build_device(dC.data_ptr(), docc.data_ptr(), dham.data_ptr(), dsum.data_ptr()),
                         args.steps)
        finally:
            ctx.close()
            del dC, docc, dham, dsum
            torch.cuda.empty_cache()

    def time_set(mols, chunk):
        # the contexts' own chunk buffers stay small (the set does not use them); the set's chunk is tuned
        ctxs = [lib.Context(m, precision="mixed", weighted=False, max_chunk_points=4096, screen_threshold=1e-10)
                for m in mols]
        dC = [torch.from_numpy(m.c_fortran()).cuda() for m in mols]
        docc = [torch.from_numpy(m.occ_fortran()).cuda() for m in mols]
        dham = [torch.zeros(m.xc_length, dtype=torch.float64, device="cuda") for m in mols]
        dsum = [torch.zeros(2, dtype=torch.float64, device="cuda") for m in mols]
        try:
            with lib.Batch(ctxs, [t.data_ptr() for t in dC], [t.data_ptr() for t in docc],
                           [t.data_ptr() for t in dham], [t.data_ptr() for t in dsum], max_chunk_points=chunk) as b:
                return timer(b.run, args.steps)
        except lib.PgxcError:
            return None
        finally:
            for c in ctxs:
                c.close()
            torch.cuda.empty_cache()

    entries = {}
    report = {}
    for cfg in (1, 2):
        c = cases.config(cfg)
        for prec in ("mixed", "fp64"):
            key, t, b = tune_single(c, prec, time_build)
            entries[key] = {"max_chunk_points": b, "ms": t[b], "workload": c.name}
            report[key] = t
    mols = cases.molecule_set(args.set_size)
    key, t, b = tune_set(mols, time_set)
    entries[key] = {"max_chunk_points": b, "ms": t[b], "workload": f"{len(mols)} molecules"}
    report[key] = t
    write(entries, args.out, torch.cuda.get_device_name(0))
    print(json.dumps({"entries": entries, "timings_ms": {k: {str(a): b for a, b in v.items()} for k, v in
                                                         report.items()}}))


if __name__ == "__main__":
    _run()
