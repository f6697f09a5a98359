"""Write noise_tables.h from the reference's noise.cc (run where the
reference sources are present; the header is committed):

    python gen_noise_tables.py <reference>/src/yafraycore/noise.cc

(or with the reference's root directory in the YR_REFERENCE environment
variable and no argument).

Blender's noise tables, as yafray 0.0.9 keeps them in noise.cc:
  hashpntf[768]  feature point offsets of the voronoi / cell bases
                 (noise.cc:7-116, indexed by HASHPNT, noise.cc:6)
  hashvectf[768] gradient vectors of blenderNoise_t (noise.cc:129-187)
The other two tables of noise.cc are periodic copies checked here:
stdp_p[514] (noise.cc:189-198) is hash[i % 256] and stdp_g[514][3]
(noise.cc:200-372) is hashvectf[3 * (i % 256) + k].  The 256-entry
permutation itself lives beside the improved Perlin noise.

The literals are written as they stand in the source (double literals
converted to float by the initialiser), so each float equals the
reference's.
"""
import os
import re
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "noise_tables.h")


def table(src, name):
    m = re.search(r"static\s+(?:unsigned char|float)\s+" + re.escape(name) + r"\s*\[[^=]*=\s*\{(.*?)\};", src, re.S)
    body = m.group(1).replace("{", " ").replace("}", " ")
    return [t.strip() for t in body.split(",") if t.strip()]


def main(src_path=None):
    if src_path is None:
        root = os.environ.get("YR_REFERENCE")
        if not root:
            sys.exit("usage: gen_noise_tables.py <path of the reference's noise.cc> (or set YR_REFERENCE)")
        src_path = os.path.join(root, "src", "yafraycore", "noise.cc")
    src = open(src_path).read()
    hp, h, hv = table(src, "hashpntf"), table(src, "hash"), table(src, "hashvectf")
    sp, sg = table(src, "stdp_p"), table(src, "stdp_g")
    assert len(hp) == 768 and len(hv) == 768 and len(h) == 512 and len(sp) == 514 and len(sg) == 1542
    hi = [int(t, 16) for t in h]
    assert all(hi[i] == hi[i % 256] for i in range(512))
    assert all(int(sp[i], 16) == hi[i % 256] for i in range(514))
    assert all(float(sg[i]) == float(hv[i % 768]) for i in range(1542))

    def rows(vals, per=8):
        return ", \\\n    ".join(", ".join(vals[i:i + per]) for i in range(0, len(vals), per))

    with open(OUT, "w") as f:
        f.write("// Generated by gen_noise_tables.py from yafray 0.0.9 noise.cc; do not edit.\n")
        f.write("// Blender's noise tables: feature point offsets of the voronoi and cell\n")
        f.write("// bases (hashpntf, noise.cc:7-116) and the gradient vectors of the blender\n")
        f.write("// and standard Perlin bases (hashvectf, noise.cc:129-187; stdp_g repeats\n")
        f.write("// it with period 256).  Initialiser lists, so that device and host\n")
        f.write("// tables can be defined from one source.\n")
        f.write("#pragma once\n\n")
        f.write("#define YR_HASHPNT_INIT { \\\n    " + rows(hp) + " }\n\n")
        f.write("#define YR_HASHVECT_INIT { \\\n    " + rows(hv) + " }\n")
    print(OUT)


if __name__ == "__main__":
    main(*sys.argv[1:])
