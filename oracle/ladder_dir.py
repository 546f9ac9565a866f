"""Test infrastructure: write the reference codec's ladder directory.

The reference DvcDec opens ``LDPCA_LadderFile/RegDecoder{1584,6336}.lad`` and
``LDPCA_LadderFile/Inverse_Matrix_H_Reg{1584,6336}.bin`` relative to its working
directory (DvcDec/src/main.cpp:82-83).  This expands the committed compact ladder
data (dvc_b200/ladders/ldpca_ladders.bin) into those files, including the CIF
pair that the reference does not ship, so that oracle/_ref/DvcDec can decode
both QCIF and CIF streams.  The encoder ladders ``RegEncoder{1584,6336}.lad``
that oracle/_ref/DvcEnc opens (DvcEnc/src/main.cpp:61-64) are written too.

    python oracle/ladder_dir.py <out_dir>     -> <out_dir>/LDPCA_LadderFile/...
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "dvc_b200", "ladders"))
import ladders as lad  # noqa: E402


def write_ladder_dir(out_dir):
    d = os.path.join(out_dir, "LDPCA_LadderFile")
    os.makedirs(d, exist_ok=True)
    for L in lad.read_compact(os.path.join(ROOT, "dvc_b200", "ladders", "ldpca_ladders.bin")):
        n = L["N"]
        enc_path = os.path.join(d, f"RegEncoder{n}.lad")
        if not os.path.exists(enc_path):
            with open(enc_path, "w") as f:
                f.write(f"{n} {L['E']}\n" + " ".join(map(str, L["jc"])) + "\n"
                        + " ".join(map(str, L["ir_full"])) + "\n")
        lad_path = os.path.join(d, f"RegDecoder{n}.lad")
        inv_path = os.path.join(d, f"Inverse_Matrix_H_Reg{n}.bin")
        if not os.path.exists(lad_path):
            lad.write_reference_lad(lad_path, lad.expand(L))
        if not os.path.exists(inv_path):
            inv = lad.gf2_inverse(lad.full_rate_h(L))
            with open(inv_path, "wb") as f:
                f.write(lad.inverse_to_reference_bin(inv))
    return d


if __name__ == "__main__":
    print(write_ladder_dir(sys.argv[1]))
