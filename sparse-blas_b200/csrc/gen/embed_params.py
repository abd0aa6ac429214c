"""Writes the trained selector parameters (a .npy of SBB_MLP_PARAMS float32)
as a C array for libsbb, so SBB_KERNEL_LEARNED plans need no file at run
time.  Build step: python3 embed_params.py <params.npy> <out.inc>."""
import sys

import numpy as np

P = np.load(sys.argv[1]).astype(np.float32).ravel()
assert P.shape == (5406,), P.shape
with open(sys.argv[2], "w") as f:
    f.write("// generated from %s by embed_params.py\n" % sys.argv[1].split("/")[-1])
    f.write("static const float kLearnedParams[%d] = {\n" % len(P))
    for i in range(0, len(P), 6):
        f.write("    " + ", ".join("%.9ef" % v for v in P[i:i + 6]) + ",\n")
    f.write("};\n")
