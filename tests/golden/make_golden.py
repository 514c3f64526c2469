"""Generate tests/golden/mggeomel.json from the reference's element tables.

Reads the reference's src/MGGeomEl.C (Hex27 family, DIMENSION 2 and 3 blocks): the
prolongation embedding matrices _embedding_matrix_q / _embedding_matrix_l (float
constants), the side topology _surf_top and the linear-in-quadratic element map Prol;
and from src/MGMesh.C (MGMesh::print_conn_lin_hf5) the split of a Quad9 / Hex27 into its
linear sub-cells for output.  These are the reference's own numbers the restated
prolongation/restriction, boundary loops and output must reproduce.

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
    "quad9_prol": ("Prol[9*4]", (9, 4)),
    "hex27_prol": ("Prol[27*8]", (27, 8)),
}
# case label of MGMesh::print_conn_lin_hf5 -> (key, sub-cells, corners)
CONN_LIN = {"9": ("quad9_conn_lin", 4, 4), "27": ("hex27_conn_lin", 8, 8)}
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
        blk = re.sub(r"//[^\n]*", "", re.sub(r"/\*.*?\*/", "", block_after(src, decl), flags=re.S))
        vals = [float(v) for v in NUM.findall(blk)]
        n = 1
        for s in shape:
            n *= s
        if len(vals) != n:
            raise ValueError("%s: %d values, expected %d" % (key, len(vals), n))
        if "surf_top" in key:
            vals = [int(v) for v in vals]
        out[key] = {"shape": shape, "data": vals}
    mesh = open(os.path.join(REF, "src", "MGMesh.C")).read()
    fn = mesh[mesh.index("void MGMesh::print_conn_lin_hf5"):]
    for label, (key, nsub, ncorner) in CONN_LIN.items():
        case = fn[re.search(r"case\s+%s\s*:" % label, fn).end():]
        case = re.sub(r"//[^\n]*", "", case[:case.index("break;")])
        tab = [[None] * ncorner for _ in range(nsub)]
        for a, b, v in re.findall(r"conn\[(\d+)\]\[(\d+)\]\s*=\s*(\d+)", case):
            tab[int(a)][int(b)] = int(v)
        if any(v is None for r in tab for v in r):
            raise ValueError(key)
        out[key] = {"shape": (nsub, ncorner), "data": [v for r in tab for v in r]}
    out["source"] += "; src/MGMesh.C (print_conn_lin_hf5)"
    with open(OUT, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
