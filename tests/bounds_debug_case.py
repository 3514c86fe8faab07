"""Run by tests/test_bounds_debug.py in a process of its own with IPR_B200_BOUNDS_CHECK=1, so
that the package binds the bounds-checked debug library (libipr_b200_dbg.so).  Prints one
JSON line: exactness of batch and single answers against the oracle, the reports of a clean
run, of the launch-argument range check on a real allocation, and of a fold launch told that
its packing-output buffer ends one polynomial early (its index checks trip on allocated
memory, so no access leaves the buffer)."""
import importlib.util
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_package():
    d = os.path.join(ROOT, "inspire-rs_b200")
    spec = importlib.util.spec_from_file_location("inspire_rs_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["inspire_rs_b200"] = m
    spec.loader.exec_module(m)
    return m


def main():
    pkg = load_package()
    import oracle as orc
    import torch
    N = 2048
    out = {"build": pkg.bounds_checked_build(), "library": os.path.basename(pkg._LIB_PATH)}
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    sdb = orc.SynthDB(plan.db_rows, plan.instances, plan.interp, plan.c, seed=7)
    qs = [orc.synth_query(300 + i, plan.db_rows, 2) for i in range(5)]
    want = [orc.respond(sdb, q) for q in qs]
    with pkg.KeywordServer.synthetic(plan, seed=7) as srv:
        got = srv.respond_batch(qs)
        single = srv.respond_to_serialized_query(qs[0])
        out["exact"] = got == want and single == want[0]
        out["clean"] = list(pkg.bounds_report())
        t = torch.empty(64 << 20, dtype=torch.uint8, device="cuda")
        out["inside"] = pkg.debug_check_extent(t.data_ptr(), t.numel())
        out["outside"] = pkg.debug_check_extent(t.data_ptr(), t.numel() + (4 << 20) + 1)
        out["host_report"] = list(pkg.bounds_report())
        pkg.debug_cut_fold_extent(N)
        try:
            cut = srv.respond_batch(qs)
        finally:
            pkg.debug_cut_fold_extent(0)
        out["cut_report"] = list(pkg.bounds_report())
        out["cut_last_differs"] = cut[-1] != want[-1]
        out["cut_others_equal"] = cut[:-1] == want[:-1]
        out["again_exact"] = srv.respond_batch(qs) == want
        out["final"] = list(pkg.bounds_report())
    print(json.dumps(out))


if __name__ == "__main__":
    main()
