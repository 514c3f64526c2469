"""Generate tests/golden/mggeomel.json from the reference's element tables.

Reads the reference's src/MGGeomEl.C (Hex27 family, DIMENSION 2 and 3 blocks): the
prolongation embedding matrices _embedding_matrix_q / _embedding_matrix_l (float
constants) and the side topology _surf_top.  These are the reference's own numbers
the restated prolongation/restriction and boundary loops must reproduce.

    python tests/golden/make_golden.py path/to/reference
    EXFEMUS_REFERENCE=path/to/reference python tests/golden/make_golden.py

The reference tree is only needed to regenerate the fixture; tests read the JSON.
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EXFEMUS_REFERENCE", "")
if not REF or not os.path.isdir(REF):
    sys.exit("make_golden.py: give the reference tree as the argument or in EXFEMUS_REFERENCE")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mggeomel.json")

TABLES = {
    "quad9_embedding_q": ("_embedding_matrix_q[4][9][9]", (4, 9, 9)),
    "quad4_embedding_l": ("_embedding_matrix_l[4][4][4]", (4, 4, 4)),
    "quad9_surf_top": ("_surf_top[12]", (4, 3)),
    "hex27_embedding_q": ("_embedding_matrix_q[8][27][27]", (8, 27, 27)),
    "hex8_embedding_l": ("_embedding_matrix_l[8][8][8]", (8, 8, 8)),
    "hex27_surf_top": ("_surf_top[54]", (6, 9)),
}
NUM = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?")


def block_after(text, decl):
    i = text.index("MGGeomEl::" + decl)
    j = text.index("{", text.index("=", i))
    depth = 0
    for k in range(j, len(text)):
        if text[k] == "{":
            depth += 1
        elif text[k] == "}":
            depth -= 1
            if depth == 0:
                return text[j:k + 1]
    raise ValueError(decl)


def main():
    src = open(os.path.join(REF, "src", "MGGeomEl.C")).read()
    out = {"source": "src/MGGeomEl.C (ELTYPE 27 blocks)"}
    for key, (decl, shape) in TABLES.items():
        blk = re.sub(r"//[^\n]*", "", block_after(src, decl))
        vals = [float(v) for v in NUM.findall(blk)]
        n = 1
        for s in shape:
            n *= s
        if len(vals) != n:
            raise ValueError("%s: %d values, expected %d" % (key, len(vals), n))
        if "surf_top" in key:
            vals = [int(v) for v in vals]
        out[key] = {"shape": shape, "data": vals}
    with open(OUT, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
