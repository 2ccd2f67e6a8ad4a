#!/usr/bin/env python3
"""Generates vp9_tables.h: the constant tables of the VP9 specification.

The tables (default probabilities, scans, quantiser lookups, subpixel filter
taps, block-size lookups) are specification data (VP9 Bitstream & Decoding
Process Specification v0.6/v0.7, sections 6, 8 and 10). The reference crate
safewords/rivet-vp9 keeps them, transcribed from the specification, in
`src/tables.rs`; this script re-emits that data as C arrays so that the host
parser, the encoder and the oracle share one copy of the numbers. Only
numbers are taken: names are prefixed `vp9t_` and the element types mapped to
fixed-width C types.

Usage: python gen_tables.py <path to rivet-vp9's src/tables.rs> <out.h>
"""
import re
import sys

TYPE_MAP = {"u8": "uint8_t", "u16": "uint16_t", "i8": "int8_t", "i32": "int32_t", "u32": "uint32_t"}


def parse_type(t, aliases):
    """Parses a Rust array type like [[u8; 3]; 16] into (ctype, [16, 3])."""
    t = t.strip()
    if t in aliases:
        return aliases[t]
    dims = []
    while t.startswith("["):
        inner, n = t[1:-1].rsplit(";", 1)
        dims.append(int(n.strip()))
        t = inner.strip()
    return TYPE_MAP[t], dims


def main():
    src, out = sys.argv[1], sys.argv[2]
    text = open(src).read()
    aliases = {}
    for m in re.finditer(r"pub\(crate\) type (\w+) = ([^;]+(?:;[^;=]+)*?);\n", text):
        aliases[m.group(1)] = parse_type(m.group(2), aliases)
    lines = [
        "/* Generated by gen_tables.py from the specification tables of the VP9",
        " * Bitstream & Decoding Process Specification (sections 6, 8, 10) as kept",
        " * in rivet-vp9 src/tables.rs. Data only; do not edit by hand. */",
        "#pragma once",
        "#include <stdint.h>",
        "",
    ]
    pat = re.compile(r"pub\(crate\) static (\w+): (.+?) = (\[.*?\]);\n", re.S)
    count = 0
    for m in pat.finditer(text):
        name, ty, body = m.group(1), m.group(2), m.group(3)
        ctype, dims = parse_type(ty, aliases)
        cbody = body.replace("[", "{").replace("]", "}")
        dimstr = "".join(f"[{d}]" for d in dims)
        lines.append(f"static const {ctype} vp9t_{name.lower()}{dimstr} = {cbody};")
        lines.append("")
        count += 1
    open(out, "w").write("\n".join(lines))
    print(f"{count} tables -> {out}")


if __name__ == "__main__":
    main()
