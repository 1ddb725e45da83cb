"""Regenerates bases.json (STO-3G, 6-31G, 6-31G* for H..Ne) from the reference's
Gaussian-format basis files (basis/STO-3G, basis/6-31G, basis/6-31GP), parsed by
dollarstorescf_b200.basis.parse_basis_text.  The JSON keeps the file's exponents
and unnormalised contraction coefficients, SP shells already split into S then P.

Usage: python -m dollarstorescf_b200.data.make_bases [reference_basis_dir]
"""
import json
import os
import sys

from dollarstorescf_b200.basis import parse_basis_text


def main(src_dir: str) -> None:
    out = {}
    for name in ("STO-3G", "6-31G", "6-31GP"):
        with open(os.path.join(src_dir, name)) as f:
            bs = parse_basis_text(f.read(), name)
        out[name] = {str(z): [{"l": s.l, "exps": s.exps, "coefs": s.coefs} for s in shells]
                     for z, shells in sorted(bs.elements.items()) if z <= 10}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bases.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else
         os.path.join(os.environ.get("DSS_REFERENCE_ROOT", "/root/reference"), "basis"))
