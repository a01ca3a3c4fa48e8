"""Fixtures from the reference's own CUDA kernels: tests/golden/ref_kernels.npz.

Three steps, because the reference exists only in the build container and the kernels only run
on a GPU:
  write : (build container) builds oracle/_ref/ref_stage_runner{,_2t} from the reference sources
          (oracle/ref_gpu_build.py) and writes one input directory per case of tests/refcases.py
          (setup.txt, grid, boundary files, the reference's chemistry data files, state.bin,
          task.txt) under --work.
  run   : (GPU machine) runs the runner on every case directory and copies each out.bin to --out.
  pack  : reads the dumps and writes the fixture (cases without a new dump keep the entries the
          fixture already has): for every case its definition,
          the digest of its initial state, the reference state the kernels read, the residual dq of
          the first stage and the conservative variables, temperature (and T_ve) after the last
          stage on the interior nodes, and for the Sod run its time-step history.  Cases flagged
          `plt` also leave the reference's own flowfield file of their final state
          (tests/golden/plt/<case>.plt, written by its FieldIO).
Usage:
  python tests/golden/make_ref_kernels.py write --work DIR [--ref REFDIR]
  python tests/golden/make_ref_kernels.py run --work DIR --out OUTDIR
  python tests/golden/make_ref_kernels.py pack --work DIR --out OUTDIR
The reference directory comes from --ref, else oracle/ref_build.py's reference_dir().
"""
import argparse
import importlib.util
import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "corefl-cpc_b200"))
sys.path.insert(0, os.path.join(REPO, "tests"))

import numpy as np  # noqa: E402

import refcases  # noqa: E402

FIXTURE = os.path.join(HERE, "ref_kernels.npz")
PLT_DIR = os.path.join(HERE, "plt")


def _runner(family):
    return os.path.join(REPO, "oracle", "_ref", "ref_stage_runner" + ("_2t" if family in ("air5", "c5") else ""))


def cmd_write(args):
    spec = importlib.util.spec_from_file_location("ref_gpu_build", os.path.join(REPO, "oracle", "ref_gpu_build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    ref = mod.reference_dir(args.ref)
    if not ref:
        sys.exit("reference sources not found: pass --ref or set COREFL_REFERENCE")
    if not args.no_build:
        print(mod.build(ref, jobs=16))
    dpath = os.path.join(args.work, "digests.json")
    digests = {}
    if args.only and os.path.exists(dpath):  # rewriting some cases keeps the others' digests
        with open(dpath) as f:
            digests = json.load(f)
    for c in refcases.CASES:
        if args.only and c["name"] not in args.only.split(","):
            continue
        d = os.path.join(args.work, c["name"])
        if c["family"] == "c5":
            digests[c["name"]] = refcases.write_reference_multi(c, d, ref)
        else:
            digests[c["name"]] = refcases.write_reference_case(c, d, ref)
        print("wrote", d)
    with open(dpath, "w") as f:
        json.dump(digests, f, indent=1)


def cmd_run(args):
    os.makedirs(args.out, exist_ok=True)
    names = sorted(n for n in os.listdir(args.work) if os.path.isdir(os.path.join(args.work, n)))
    if args.only:
        names = [n for n in names if n in args.only.split(",")]
    for n in names:
        c = refcases.case_by_name(n)
        d = os.path.abspath(os.path.join(args.work, n))
        r = subprocess.run([_runner(c["family"]), d], capture_output=True, text=True, timeout=args.timeout)
        os.makedirs(os.path.join(args.out, n), exist_ok=True)
        with open(os.path.join(args.out, n, "log.txt"), "w") as f:
            f.write(r.stdout[-20000:] + "\n---- stderr\n" + r.stderr[-20000:])
        if r.returncode != 0:
            # a CUDA error ends the whole run; a host-side failure (a setup the reference refuses)
            # only skips the case
            if "CUDA error" in r.stderr:
                sys.exit("runner hit a CUDA error on %s: %s" % (n, r.stderr[-2000:]))
            print("runner failed on %s (rc %d): %s" % (n, r.returncode, r.stderr[-500:]))
            continue
        os.replace(os.path.join(d, "out.bin"), os.path.join(args.out, n, "out.bin"))
        plt = os.path.join(d, "output", "flowfield.plt")
        if os.path.exists(plt):
            os.replace(plt, os.path.join(args.out, n, "flowfield.plt"))
        if os.path.exists(os.path.join(d, "ref_metric.bin")):
            os.replace(os.path.join(d, "ref_metric.bin"), os.path.join(args.out, n, "ref_metric.bin"))
        print(n, r.stdout.strip().splitlines()[-1] if r.stdout.strip() else "")


def cmd_pack(args):
    with open(os.path.join(args.work, "digests.json")) as f:
        digests = json.load(f)
    arrays = {}
    meta = {}
    if os.path.exists(FIXTURE):  # cases without a new dump keep their entries
        old = np.load(FIXTURE)
        meta = json.loads(bytes(old["meta"]).decode())
        arrays = {k: old[k] for k in old.files if k != "meta"}
    for c in refcases.CASES:
        n = c["name"]
        path = os.path.join(args.out, n, "out.bin")
        if not os.path.exists(path):
            print("no new dump for", n, "(kept)" if n in meta else "(missing)")
            continue
        for k in [k for k in arrays if k.startswith(n + "/")]:
            del arrays[k]
        plt = os.path.join(args.out, n, "flowfield.plt")
        if os.path.exists(plt):  # the reference's flowfield file: tests/golden/plt/<case>.plt
            os.makedirs(PLT_DIR, exist_ok=True)
            shutil.copy(plt, os.path.join(PLT_DIR, n + ".plt"))
        d = refcases.read_dump(path)
        blk = d["blocks"][0]
        g = blk["dims"][3]
        meta[n] = dict(case=c, digest=digests[n], rho_inf=d["rho_inf"], v_inf=d["v_inf"], p_inf=d["p_inf"],
                       speed_of_sound=d["speed_of_sound"], steps=d["steps"], time=d["time"], dt=d["dt"])
        if c["family"] == "sod":
            j = blk["dims"][1] // 2
            arrays[n + "/cv"] = blk["cv"][:, g, g + j, g:-g]
            arrays[n + "/dts"] = d["dts"]
        elif c["family"] == "c5":
            nb = len(d["blocks"])
            for b, bk in enumerate(d["blocks"]):
                arrays[n + "/dq0/%d" % b] = d["dq"][b]
                arrays[n + "/cv/%d" % b] = refcases.interior(bk["cv"], g)
                arrays[n + "/T/%d" % b] = refcases.interior(bk["bv"], g)[5]
                arrays[n + "/Tve/%d" % b] = refcases.interior(bk["temperature_ve"], g)[0]
            meta[n]["n_block"] = nb
            # the reference Mesh's own metric and Jacobian of every padded node (before the runner
            # loaded the case's), which pin the host grid module that computes them here
            mp = os.path.join(args.out, n, "ref_metric.bin")
            if os.path.exists(mp):
                raw = np.fromfile(mp, dtype="<f8")
                arrays[n + "/ref_metric"] = raw
        else:
            arrays[n + "/dq0"] = d["dq"][0]
            arrays[n + "/cv"] = refcases.interior(blk["cv"], g)
            arrays[n + "/T"] = refcases.interior(blk["bv"], g)[5]
            if "temperature_ve" in blk:
                arrays[n + "/Tve"] = refcases.interior(blk["temperature_ve"], g)[0]
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(FIXTURE, **arrays)
    print("wrote", FIXTURE, "with", len(meta), "cases")


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    w = sub.add_parser("write")
    w.add_argument("--work", required=True)
    w.add_argument("--ref", default=None)
    w.add_argument("--only", default=None)
    w.add_argument("--no-build", action="store_true")
    r = sub.add_parser("run")
    r.add_argument("--work", required=True)
    r.add_argument("--out", required=True)
    r.add_argument("--only", default=None)
    r.add_argument("--timeout", type=float, default=600)
    p = sub.add_parser("pack")
    p.add_argument("--work", required=True)
    p.add_argument("--out", required=True)
    a = ap.parse_args()
    {"write": cmd_write, "run": cmd_run, "pack": cmd_pack}[a.cmd](a)


if __name__ == "__main__":
    main()
