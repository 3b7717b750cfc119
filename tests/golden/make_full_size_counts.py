"""Write tests/golden/full_size_counts.json: counts at full size computed by
the reference's own generated search kernel (baseline/refgen.py: KernelGen
output with warpCentric, warpBalancing and tailExpansion on, built for
sm_100a), for the cases the oracle cannot finish in seconds:

  * the 4-cycle 0->1->2->3->0 on the 2.6M-node / 36M-edge graph, delta 86400;
  * the 16 queries of the 64-query batch mix in everest_b200.workloads.BATCH_SLICE,
    over every root of the same graph.

Needs a GPU and the built generated kernels (python -m baseline.refgen build);
run from the repository root:

    python tests/golden/make_full_size_counts.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from baseline import refgen as R  # noqa: E402
from everest_b200 import synth, workloads  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    spec = synth.SPECS["bursty-2.6m-36m"]
    u, v, t = synth.load_or_generate(spec.name)
    rg = R.RefGraph.from_oracle_graph(O.Graph(u, v, t, spec.num_nodes))
    out = {"source": "the reference's generated search kernel (KernelGen with warpCentric, warpBalancing and "
                     "tailExpansion on, built for sm_100a by baseline/refgen.py) on a B200; this library's "
                     "counts are equal (tests/test_gpu_refgen.py); regenerate with "
                     "tests/golden/make_full_size_counts.py on a GPU box",
           spec.name: {}}
    c, _ = R.count(rg, [0, 1, 2, 3], [1, 2, 3, 0], 86400)
    out[spec.name]["4-cycle delta 86400"] = c
    out[spec.name]["batch slice"] = {}
    for q in workloads.refgen_batch_slice():
        c, _ = R.count(rg, q["mu"], q["mv"], q["delta"])
        out[spec.name]["batch slice"][q["name"]] = {"mu": q["mu"], "mv": q["mv"], "delta": q["delta"], "count": c}
    rg.free()
    with open(os.path.join(HERE, "full_size_counts.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
