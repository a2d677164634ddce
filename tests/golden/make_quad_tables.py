"""Generate tests/golden/quad_tables.json from the reference source.

Reads the 64- and 128-node t quadrature tables (t_val / w_val) of
gauss_legendre_points (src/module/precompute_t.f90:484-895) as text, exactly
as written in the reference, so the oracle's table rules and the fast-quad
self-check can use the reference's own nodes and weights.

Run where the reference tree is present (it is not on the GPU box), with the
root of the reference project as the one required argument:
    python tests/golden/make_quad_tables.py <reference-root>
"""
import json
import os
import re
import sys


def main(ref_root: str) -> None:
    src = open(os.path.join(ref_root, "src", "module", "precompute_t.f90")).read()
    body = src[src.index("subroutine gauss_legendre_points"):]
    body = body[:body.index("end subroutine gauss_legendre_points")]
    blocks = re.findall(r"(t_val|w_val)\s*=\s*\[(.*?)\]", body, re.S)
    out = {}
    for name, text in blocks:
        vals = [float(x.replace("d", "e").replace("D", "e")) for x in re.findall(r"[-0-9.]+[dD][-+0-9]+", text)]
        out.setdefault(str(len(vals)), {})[name] = vals
    assert set(out) == {"64", "128"}, out.keys()
    out["source"] = "src/module/precompute_t.f90:484-895 (gauss_legendre_points), values as written"
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "quad_tables.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_quad_tables.py <reference-root>")
    main(sys.argv[1])
