"""Records golden fixtures from the REFERENCE's own kernels (cudaLJ.cu built
from source into oracle/_ref/libljref.so) run on a GPU.

    python tests/golden/make_golden.py [out_dir]      (default: tests/golden)

For each case of refcases.CASES it stores the inputs and the reference's
outputs: counts, prefix (offsets), the per-cell index sets in ascending order,
the candidate-pair count of ComputeNbInteractions and the compat energies of
ComputeParticleInterationsParPartNoLoop indexed by original particle.  The CPU
suite (tests/test_golden.py) checks the oracle against these files."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import ljoracle as O  # noqa: E402
import refcases  # noqa: E402


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    for name, make in refcases.CASES.items():
        (x, y, z), box, cutoff = make()
        r = O.ref_run(x, y, z, box, cutoff)
        v_by_index = np.empty(len(x), np.float32)
        v_by_index[r.index] = r.v
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), x=x, y=y, z=z, box=np.float32(box),
                            cutoff=np.float32(cutoff), counts=r.counts, prefix=r.prefix,
                            index_sorted=refcases.sorted_within_cells(r.index, r.prefix),
                            nbinter=np.uint64(r.nbinter), v_by_index=v_by_index)
        print(name, len(x), "cells", len(r.counts), "candidates", r.nbinter)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
