"""Build recipe for the compiled-reference checker (TEST INFRASTRUCTURE).

Plays the role of the SDDS ``nlpp`` code generator, which is not in the
reference tree: it reads the reference's namelist definition files
(``src/*.nl``, e.g. integrate.nl:8-25) and writes one C header per file that
declares each namelist variable with its default and a NAMELIST table in the
layout of oracle/shim/namelist.h.  The reference includes these headers inside
its setup functions (integrate.c:47, cathode.c:27, geometry.c:25) or at file
scope (poisson_correction.c:16), so every variable is ``static``.

Usage: python gen_nl_headers.py <reference src dir> <output dir>
"""
import os
import re
import sys

TYPES = {
    "double": ("double", "NL_DOUBLE", "0"),
    "long": ("long", "NL_LONG", "0"),
    "int": ("int", "NL_INT", "0"),
    "int32_t": ("int32_t", "NL_INT", "0"),
    "short": ("short", "NL_SHORT", "0"),
    "STRING": ("STRING", "NL_STRING", "NULL"),
}

DECL = re.compile(r"^\s*(double|long|int32_t|int|short|STRING)\s+(\w+)\s*(=\s*([^;]+))?;")


def parse(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    groups, cur = [], None
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("#namelist"):
            cur = [s.split()[1], []]
            groups.append(cur)
        elif s.startswith("#end"):
            cur = None
        elif cur is not None:
            m = DECL.match(s)
            if m:
                cur[1].append((m.group(1), m.group(2), (m.group(4) or "").strip()))
    return groups


def emit(groups, guard):
    out = [f"/* generated from the reference's {guard}.nl by oracle/gen_nl_headers.py */",
           '#include "namelist.h"', "#include <stdint.h>"]
    for name, decls in groups:
        items = []
        for ctype, var, default in decls:
            c, kind, zero = TYPES[ctype]
            out.append(f"static {c} {var} = {default or zero};")
            items.append(f'{{"{var}", {kind}, (void *)&{var}}}')
        out.append(f"static NL_ITEM {name}_items[] = {{{', '.join(items)}}};")
        out.append(f'static NAMELIST {name} = {{{name}_items, "{name}", {len(items)}}};')
        if name == "point":
            out.append("static NAMELIST_TEXT namelist_text;")
    return "\n".join(out) + "\n"


def main(src, dst):
    os.makedirs(dst, exist_ok=True)
    for fn in sorted(os.listdir(src)):
        if fn.endswith(".nl"):
            base = fn[:-3]
            with open(os.path.join(src, fn)) as f:
                groups = parse(f.read())
            with open(os.path.join(dst, base + ".h"), "w") as f:
                f.write(emit(groups, base))


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
