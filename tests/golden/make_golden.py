"""Generates the golden fixtures of this directory from the reference sources.

Run where the reference TAL-SH tree sits beside the repository (../reference
relative to the repository root; TALSH_REFERENCE overrides):
python tests/golden/make_golden.py
The fixtures are committed; nothing at test time reads the reference.

  tensor_contractions.json  the 48 benchmark patterns and shapes of the
                            reference's tensor_contractions.txt (read by
                            main.F90:912-1026), verbatim.
  patterns.json             digital forms and matricizations that the
                            reference states in its sources and tests:
                            test.cpp's hand-written digital pattern of
                            test_nvtal_c, the constant-input contraction of
                            test_talsh_c, the nwchem pattern, and the C1
                            matricizations that follow from
                            tensor_algebra_cpu.F90:5757-5956 (CPU) and
                            :5613-5755 (GPU variant).
"""
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("TALSH_REFERENCE") or os.path.normpath(os.path.join(HERE, "..", "..", "..", "reference"))


def contractions():
    path = os.path.join(REF, "tensor_contractions.txt")
    lines = [ln.rstrip("\n") for ln in open(path) if ln.strip()]
    out = []
    for i in range(0, len(lines) - 1, 2):
        pat = lines[i].strip()
        nums = [int(x) for x in lines[i + 1].split()]
        shapes = []
        k = 0
        for _ in range(3):
            r = nums[k]
            shapes.append(nums[k + 1:k + 1 + r])
            k += 1 + r
        out.append({"pattern": pat, "D": shapes[0], "L": shapes[1], "R": shapes[2]})
    return out


def stated_patterns():
    test_cpp = open(os.path.join(REF, "test.cpp")).read()
    m = re.search(r"int cptrn0\[\]=\{([^}]*)\}", test_cpp)
    nvtal = [int(x) for x in m.group(1).split(",")]
    m2 = re.search(r'talshTensorContract\("(D\(a,b,i,j\)\+=L\(c,b,d,a\)\*R\(j,d,i,c\))"', test_cpp)
    m3 = re.search(r'talshTensorContract\("(D\(a,b\)\+=L\(c,d\)\*R\(d,a,b,c\))"', test_cpp)
    return {
        # test_nvtal_c passes this digital pattern to gpu_tensor_block_contract_dlf
        # for 40^4 tensors; its symbolic twin is D(a,b,c,d)+=L(d,c,i,j)*R(b,a,i,j).
        "nvtal_digital": {"pattern": "D(a,b,c,d)+=L(d,c,i,j)*R(b,a,i,j)", "digital": nvtal,
                          "drank": 4, "lrank": 4, "rrank": 4},
        "talsh_c_pattern": m2.group(1),
        "nwchem_pattern": m3.group(1),
        # C1: digital form and both matricizations (1-based; dprm N2O, lprm/rprm O2N).
        "c1": {"pattern": "D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)",
               "digital": [1, -3, -1, 3, -3, 2, -2, 4],
               "cpu": {"dprm": [1, 3, 2, 4], "lprm": [3, 1, 2, 4], "rprm": [2, 3, 1, 4],
                       "ncd": 2, "nlu": 2, "nru": 2, "nhu": 0},
               "gpu": {"dprm": [1, 3, 2, 4], "lprm": [3, 2, 1, 4], "rprm": [1, 3, 2, 4],
                       "ncd": 2, "nlu": 2, "nru": 2}},
        "c1_transpose": {"pattern": "D(i,c,a,b)=L(a,b,c,i)", "digital": [3, 4, 2, 1]},
    }


if __name__ == "__main__":
    with open(os.path.join(HERE, "tensor_contractions.json"), "w") as f:
        json.dump(contractions(), f, indent=1)
    with open(os.path.join(HERE, "patterns.json"), "w") as f:
        json.dump(stated_patterns(), f, indent=1)
    print("wrote fixtures to", HERE)
