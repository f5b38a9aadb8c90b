"""Generate tests/golden/reference_tables.json from the reference's TOP_GPU.m.

Run in a container that has the reference checked out (read-only):

    python tests/golden/make_golden.py /path/to/TOP_GPU_on_matlab

The script reads TOP_GPU.m as text and extracts, as data:
  * the element stiffness closed form (FEA_VoxelBasedElementStiffnessMatrix,
    TOP_GPU.m:1465-1503): the constant vector C and the twelve 6x6 blocks,
    evaluated for nu = 0.3 with MATLAB's operation order;
  * the restriction/interpolation tables RI for span 2 and 4
    (Solving_Operator4MultiGridRestrictionAndInterpolation, TOP_GPU.m:2165-2328);
  * the sub-element node maps for span 2 and 4 (Solving_SubEleNodMat,
    TOP_GPU.m:1938-2017).
Floats are stored with float.hex() so the fixture is bit-exact.  Tests read
only the JSON; nothing at test time touches the reference.
"""
import json
import re
import sys
from pathlib import Path

import numpy as np


def _function_text(src: str, name: str) -> str:
    m = re.search(r"^function[^\n]*\b" + re.escape(name) + r"\b", src, re.M)
    if not m:
        raise KeyError(name)
    start = m.start()
    nxt = re.search(r"^function\b", src[m.end():], re.M)
    end = m.end() + nxt.start() if nxt else len(src)
    return src[start:end]


def _strip_comments(text: str) -> str:
    return "\n".join(line.split("%", 1)[0] for line in text.splitlines())


def _matrix_literal(text: str, lhs: str, occurrence: int = 0) -> str:
    """Body of `lhs = [ ... ];` (continuations joined)."""
    pat = re.compile(re.escape(lhs) + r"\s*=\s*\[(.*?)\];", re.S)
    found = pat.findall(text)
    return found[occurrence].replace("...", " ")


def _parse_rows(body: str, row_sep_newline: bool):
    rows = []
    chunks = body.split(";")
    if row_sep_newline:
        chunks = [c for part in chunks for c in part.split("\n")]
    for chunk in chunks:
        toks = chunk.split()
        if toks:
            rows.append(toks)
    return rows


def ke_closed_form(src: str, nu: float = 0.3) -> np.ndarray:
    text = _strip_comments(_function_text(src, "FEA_VoxelBasedElementStiffnessMatrix"))
    cbody = re.search(r"C\s*=\s*\[(.*?)\];", text, re.S).group(1)
    C = []
    for tok in cbody.split():
        num, den = tok.split("/") if "/" in tok else (tok, "1")
        C.append(float(num) / float(den))

    def tok_val(tok):
        m = re.fullmatch(r"(-?)C\((\d+)\)", tok)
        if m:
            v = C[int(m.group(2)) - 1]
            return -v if m.group(1) else v
        return float(tok)

    blocks = {}
    for name in ["A11", "B11", "A22", "B22", "A12", "B12", "A13", "B13", "A14", "B14", "A23", "B23"]:
        rows = _parse_rows(_matrix_literal(text, name), row_sep_newline=False)
        blocks[name] = np.array([[tok_val(t) for t in r] for r in rows], dtype=np.float64)
        assert blocks[name].shape == (6, 6), name
    ke_line = re.search(r"KE\s*=\s*1/\(1\+nu\)/\(2\*nu-1\)\*\((.*?)\);", text, re.S).group(1).replace("...", " ")
    a_lay, b_lay = re.findall(r"\[(.*?)\]", ke_line, re.S)

    def layout(lay):
        rows = _parse_rows(lay, row_sep_newline=False)
        out = []
        for r in rows:
            out.append([blocks[t.rstrip("'")].T if t.endswith("'") else blocks[t] for t in r])
        return np.block(out)

    A = layout(a_lay)
    B = layout(b_lay)
    s = 1.0 / (1.0 + nu) / (2.0 * nu - 1.0)
    return s * (A + nu * B)


def ri_table(src: str, span: int) -> np.ndarray:
    text = _strip_comments(_function_text(src, "Solving_Operator4MultiGridRestrictionAndInterpolation"))
    body = _matrix_literal(text, "ss", occurrence=0 if span == 2 else 1)
    rows = _parse_rows(body, row_sep_newline=True)
    arr = np.array([[float(t) for t in r] for r in rows], dtype=np.float64)
    assert arr.shape == ((span + 1) ** 3, 8), arr.shape
    return arr


def subele_nodmat(src: str, span: int) -> np.ndarray:
    text = _strip_comments(_function_text(src, "Solving_SubEleNodMat"))
    body = _matrix_literal(text, "val", occurrence=0 if span == 2 else 1)
    rows = _parse_rows(body, row_sep_newline=True)
    arr = np.array([[int(t) for t in r] for r in rows], dtype=np.int64)
    assert arr.shape == (span ** 3, 8), arr.shape
    return arr


def main(ref_root: str) -> None:
    src = (Path(ref_root) / "TOP_GPU.m").read_text(encoding="utf-8", errors="replace")
    out = {
        "source": "TOP_GPU.m (mnivan/TOP_GPU_on_matlab)",
        "Ke_nu0.3_cell1": [float(v).hex() for v in ke_closed_form(src).flatten(order="F")],
        "RI2": [float(v).hex() for v in ri_table(src, 2).flatten(order="F")],
        "RI4": [float(v).hex() for v in ri_table(src, 4).flatten(order="F")],
        "SUB2": subele_nodmat(src, 2).tolist(),
        "SUB4": subele_nodmat(src, 4).tolist(),
    }
    dst = Path(__file__).with_name("reference_tables.json")
    dst.write_text(json.dumps(out, indent=0))
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference checkout (the directory holding TOP_GPU.m)>")
    main(sys.argv[1])
