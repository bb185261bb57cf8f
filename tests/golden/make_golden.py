"""Regenerate the golden fixtures from trinity's own code (the reference,
compiled from its sources by ``make -C oracle ref``). Run in a container where
the reference sources exist; the GPU box only reads the committed fixtures.

  numeric_vectors.jsonl  inputs/outputs of the reference's numeric.cpp
                         (eigenDecompose, interpolateTensor, computeQuality,
                         approxRiemannDist, computeSteinerPoint), hex doubles
  ref_stage_digests.json per-stage SHA-256 of the reference's full-precision
                         state (1 thread, -ffp-contract=off, project log/exp/pow)
                         after the metric and every kernel of every round, plus
                         the SHA-256 of its Mesh::store output

    python tests/golden/make_golden.py
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from tests.oracle_lib import REF_EXACT, REF_SRC, ORACLE_DIR, digest, read_snapshot  # noqa: E402
from trinity_b200 import meshgen  # noqa: E402


# (name, generator config, grid side override, rounds)
CASES = [("c1", "c1", None, 3), ("c2_n60", "c2", 60, 2), ("c4_n50", "c4", 50, 2),
         ("c2", "c2", None, 3)]
FIXTURE_CASES = [("grid4_shock4", "examples/mesh/GRID4.mesh", "examples/solut/shock4.bb", 2, 3, 64, 1.0, 2)]


def run_ref(mesh, bb, rounds, depth, bucket, target, norm, tmp, tag):
    prefix = os.path.join(tmp, tag)
    out = prefix + ".out.mesh"
    subprocess.run([REF_EXACT, mesh, bb, str(rounds), str(depth), str(bucket), str(target), str(norm),
                    "--dump", prefix, "--out", out], check=True, stdout=subprocess.DEVNULL,
                   env=dict(os.environ, OMP_NUM_THREADS="1"))
    stages = ["load", "metric"] + [f"r{r}.{k}" for r in range(rounds)
                                   for k in ("refine", "coarse", "swap", "smooth")]
    import hashlib
    res = {"stages": {s: digest(read_snapshot(f"{prefix}.{s}.bin")) for s in stages},
           "store_sha256": hashlib.sha256(open(out, "rb").read()).hexdigest(),
           "params": dict(rounds=rounds, depth=depth, bucket=bucket, target=target, norm=norm)}
    return res


def main():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, "ref", f"REF={REF_SRC}"], check=True)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for tag, cfg, n, rounds in CASES:
            mp, bp, c = meshgen.write_config(cfg, tmp, n)
            out[tag] = run_ref(mp, bp, rounds, c["depth"], c["bucket"], c["target"], c["norm"], tmp, tag)
            out[tag]["config"] = {"name": cfg, "n": n}
            print(tag, "ok", flush=True)
        for tag, mesh, bb, rounds, depth, bucket, target, norm in FIXTURE_CASES:
            out[tag] = run_ref(os.path.join(REF_SRC, mesh), os.path.join(REF_SRC, bb), rounds, depth,
                               bucket, target, norm, tmp, tag)
            out[tag]["fixture"] = {"mesh": mesh, "bb": bb}
            print(tag, "ok", flush=True)
    json.dump(out, open(os.path.join(HERE, "ref_stage_digests.json"), "w"), indent=1)
    vec = subprocess.run([os.path.join(ORACLE_DIR, "_ref", "ref_numeric"), "64"], check=True,
                         capture_output=True, text=True).stdout
    open(os.path.join(HERE, "numeric_vectors.jsonl"), "w").write(vec)
    print("written")


if __name__ == "__main__":
    main()
