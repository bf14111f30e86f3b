"""Generate aborting definitions for symbols missing from the oracle link.

Test infrastructure for oracle/Makefile: reads the linker's
"undefined reference to `sym'" lines and writes a C++ file that defines each
missing function symbol (by its mangled name) as a function that aborts, so
that out-of-path reference files that cannot be compiled here (VTK output
writers, Eigen-heavy MathTools) do not block linking the hot path. None of
these symbols is reached by the oracle's code paths.
"""
import re
import subprocess
import sys

src, dst = sys.argv[1], sys.argv[2]
text = open(src).read()
names = sorted(set(re.findall(r"undefined reference to `([^']+)'", text)))
mangled = []
for n in names:
    if n.startswith("_Z") or re.match(r"^[A-Za-z_][A-Za-z0-9_]*$", n):
        mangled.append(n)
    else:
        # demangled form printed by the linker: recover nothing; report it
        print("gen_stubs: cannot stub demangled symbol", n, file=sys.stderr)
with open(dst, "w") as f:
    f.write("// generated by oracle/gen_stubs.py\n#include <cstdio>\n#include <cstdlib>\n")
    for i, n in enumerate(mangled):
        f.write(f'extern "C" void m2c_oracle_stub_{i}() __asm__("{n}");\n')
        f.write(f'extern "C" void m2c_oracle_stub_{i}() {{ fprintf(stderr, "oracle stub reached: {n}\\n"); abort(); }}\n')
print(f"gen_stubs: {len(mangled)} stubs")
