"""Writes vc1cu_entropy_lengths.h: the VC-1 code lengths the transform RD's bit estimates need.

The lengths are bitstream-format data (SMPTE ST 421: the eight progressive AC run/level VLC
tables and their escape codes, the P-picture CBPCY table, TTMB / TTBLK / SUBBLKPAT, the
progressive inter and intra scans, the four MVDATA tables and the bitplane IMODE / NORM-2 / NORM-6 codes). They are read from the reference tree, whose tables state them, and
only the lengths (never the code words) are kept. Run it where the reference tree is present:

    python libvc1_b200/csrc/gen_entropy_lengths.py [reference tree]    (default $LIBVC1_REFERENCE
                                                                        or /root/reference)
The output is committed; builds do not run this script.
"""
from __future__ import annotations

import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SETS = ["HighMotionIntra", "HighMotionInter", "LowMotionIntra", "LowMotionInter", "MidRateIntra", "MidRateInter",
        "HighRateIntra", "HighRateInter"]


def _ints(s):
    return [int(x, 0) for x in re.findall(r"-?(?:0x[0-9a-fA-F]+|\d+)", s)]


def _block(text, name):
    m = re.search(re.escape(name) + r"\s*(?:\[[^\]]*\])*\s*=\s*\{\{?(.*?)\}\}?;", text, re.S)
    if not m:
        raise SystemExit(f"{name} not found")
    return m.group(1)


def _gblock(text, name):
    """A std::array initialiser of the group-A tables (`name{{...}};` or `name = {{...}};`)."""
    m = re.search(r"\b" + re.escape(name) + r"\s*=?\s*\{\{(.*?)\}\};", text, re.S)
    if not m:
        raise SystemExit(f"{name} not found")
    return m.group(1)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LIBVC1_REFERENCE", "/root/reference")
    ent = open(os.path.join(ref, "src", "vc1_entropy_tables.h")).read()
    inh = open(os.path.join(ref, "src", "encoder_internal.h")).read()
    grp = open(os.path.join(ref, "src", "vc1_groupa_tables.h")).read()
    out = ["// vc1cu_entropy_lengths.h - VC-1 code lengths of the transform RD's bit estimates.",
           "// Generated by gen_entropy_lengths.py (do not edit): bitstream-format data of SMPTE ST 421",
           "// (AC run/level tables and escapes of the eight progressive coding sets, P CBPCY, TTMB,",
           "// TTBLK, SUBBLKPAT, the progressive inter and intra scans, MVDATA, IMODE, NORM-2, NORM-6); lengths",
           "// only, no code words.",
           "// The small tables' storage is VC1CU_ENT_TABLE (constexpr unless the includer puts them in",
           "// device constant memory); the AC entries are host data (dense tables are built from them).",
           "#pragma once", "", "#include <cstdint>", "", "#ifndef VC1CU_ENT_TABLE", "#define VC1CU_ENT_TABLE constexpr",
           "#endif", "", "namespace vc1cu {", "namespace ent {", ""]
    counts, rows, esc = [], [], []
    for i, s in enumerate(SETS):
        body = _block(ent, "k" + s)
        entries = re.findall(r"AcVlcEntry\{\s*(0x[0-9a-fA-F]+)u?,\s*(\d+),\s*(\d+),\s*(\d+),\s*(true|false)\s*\}", body)
        counts.append(len(entries))
        for _code, bits, run, level, last in entries:
            rows.append((i, int(run), int(level), 1 if last == "true" else 0, int(bits)))
        m = re.search(r"k" + s + r"Escape\{\s*0x[0-9a-fA-F]+u?,\s*(\d+)\s*\}", ent)
        esc.append(int(m.group(1)))
    out.append("// (coding set, run, level, last, bits) of every direct AC code, coding sets 0..7 in order:")
    out.append("// 0 high-motion intra, 1 high-motion inter, 2 low-motion intra, 3 low-motion inter,")
    out.append("// 4 mid-rate intra, 5 mid-rate inter, 6 high-rate intra, 7 high-rate inter")
    out.append(f"constexpr int kAcEntries = {len(rows)};")
    out.append("constexpr uint8_t kAcEntry[kAcEntries][5] = {")
    for k in range(0, len(rows), 6):
        out.append("    " + " ".join("{%d, %d, %d, %d, %d}," % r for r in rows[k:k + 6]))
    out.append("};")
    out.append("VC1CU_ENT_TABLE uint8_t kAcEscapeBits[8] = {" + ", ".join(map(str, esc)) + "};")
    cbp = re.findall(r"\{\s*\d+\s*,\s*(\d+)\s*\}", _block(inh, "kPcbpVlc"))
    assert len(cbp) == 64
    out.append("// P-picture CBPCY (table 0), by the six-bit CBP")
    out.append("VC1CU_ENT_TABLE uint8_t kPcbpBits[64] = {" + ", ".join(cbp) + "};")
    for name, n in (("kTtmbBits", 16), ("kTtblkBits", 8), ("kTtSymbolVariant", 8), ("kSubblkBits", 15)):
        v = _ints(_block(inh, name))
        assert len(v) == 3 * n, name
        out.append(f"VC1CU_ENT_TABLE uint8_t {name}[3][{n}] = {{" +
                   ", ".join("{" + ", ".join(map(str, v[r * n:(r + 1) * n])) + "}" for r in range(3)) + "};")
    for name, n in (("kInterScan", 64), ("kInterScan8x4", 32), ("kInterScan4x8", 32), ("kInterScan4x4", 16),
                    ("kIntraScan", 64)):
        v = _ints(_block(inh, name))
        assert len(v) == n, name
        out.append(f"VC1CU_ENT_TABLE uint8_t {name}[{n}] = {{" + ", ".join(map(str, v)) + "};")
    # picture-layer lengths of the P motion-bit estimate: MVDATA of the four MV tables, IMODE,
    # NORM-2 and NORM-6 bitplane symbols
    out.append("// MVDATA lengths of MV tables 0..3 by symbol (0..72)")
    v = _ints(_gblock(grp, "kMvDiffBits"))
    assert len(v) == 4 * 73, "kMvDiffBits"
    out.append("VC1CU_ENT_TABLE uint8_t kMvDiffBits[4][73] = {" +
               ", ".join("{" + ", ".join(map(str, v[r * 73:(r + 1) * 73])) + "}" for r in range(4)) + "};")
    out.append("// bitplane IMODE, NORM-2 and NORM-6 symbol lengths")
    for name, n in (("kImodeBits", 7), ("kNorm2Bits", 4), ("kNorm6Bits", 64)):
        v = _ints(_gblock(grp, name))
        assert len(v) == n, name
        out.append(f"VC1CU_ENT_TABLE uint8_t {name}[{n}] = {{" + ", ".join(map(str, v)) + "};")
    out += ["", "}  // namespace ent", "}  // namespace vc1cu", ""]
    path = os.path.join(HERE, "vc1cu_entropy_lengths.h")
    open(path, "w").write("\n".join(out))
    print(f"wrote {path}: {len(rows)} AC entries {counts}")


if __name__ == "__main__":
    main()
