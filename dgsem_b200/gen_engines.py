"""Generates the explicit Engine instantiation units and the runtime factory.

The fused stage kernel is a template over (dimension, nodes per direction,
volume flux, surface flux, shock capturing); each supported combination is
instantiated in its own translation unit (grouped by dimension and node count)
so nvcc can compile them in parallel.  Run by dgsem_b200/build.py.
"""
from __future__ import annotations

import os

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "generated")


def combos():
    out = set()
    # 2D Euler: every n in 2..8 with the three volume fluxes and LLF, and the
    # Hennemann-Gassner shock capturing with Chandrashekar/LLF.
    for n in range(2, 9):
        for vf in range(3):
            out.add((2, n, vf, 0, 0))
        out.add((2, n, 0, 0, 1))
    # n = 4 (the benchmark degree N = 3): every flux / shock-capturing mix.
    for vf in range(3):
        for sf in range(2):
            for hg in range(2):
                out.add((2, 4, vf, sf, hg))
    # 3D Euler (periodic): n in 2..5 with the three volume fluxes and LLF, and
    # Hennemann-Gassner shock capturing with Chandrashekar/LLF; at n = 4 with
    # every volume flux.
    for n in range(2, 6):
        for vf in range(3):
            out.add((3, n, vf, 0, 0))
        out.add((3, n, 0, 0, 1))
    for vf in range(3):
        out.add((3, 4, vf, 0, 1))
    return sorted((d, n, vf, sf, hg, 0) for (d, n, vf, sf, hg) in out) + ns_combos()


def ns_combos():
    # 2D Navier-Stokes (BR1, periodic or walls): n in 2..8, the three volume
    # fluxes, LLF; 3D Navier-Stokes (periodic): n in 2..5, the three volume
    # fluxes, LLF (node-parallel shapes).
    # 2D Navier-Stokes with Hennemann-Gassner shock capturing (the
    # reference's viscous KHI setup): Chandrashekar / LLF, n in 2..8.
    return (sorted((2, n, vf, 0, 0, 1) for n in range(2, 9) for vf in range(3)) +
            sorted((2, n, 0, 0, 1, 1) for n in range(2, 9)) +
            sorted((3, n, vf, 0, 0, 1) for n in range(2, 6) for vf in range(3)))


def generate() -> list[str]:
    os.makedirs(GEN, exist_ok=True)
    cs = combos()
    groups: dict = {}
    for c in cs:
        groups.setdefault((c[0], c[1]), []).append(c)
    files = []
    for (d, n), items in groups.items():
        path = os.path.join(GEN, f"engines_{d}d_n{n}.cu")
        lines = [f"// Generated by gen_engines.py: Engine instantiations, {d}D, n = {n}.",
                 '#include "../engine.cuh"', "namespace dgsem {"]
        for (_, _, vf, sf, hg, ns) in items:
            lines.append(f"std::unique_ptr<EngineBase> create_engine_{d}_{n}_{vf}_{sf}_{hg}_{ns}() {{")
            lines.append(f"  return std::make_unique<Engine<{d}, {n}, {vf}, {sf}, "
                         f"{'true' if hg else 'false'}, {'true' if ns else 'false'}>>();")
            lines.append("}")
        lines.append("}  // namespace dgsem")
        _write_if_changed(path, "\n".join(lines) + "\n")
        files.append(path)
    path = os.path.join(GEN, "engine_factory.cu")
    lines = ["// Generated by gen_engines.py: runtime scheme -> Engine instantiation.",
             '#include "../engine.cuh"', "namespace dgsem {"]
    for (d, n, vf, sf, hg, ns) in cs:
        lines.append(f"std::unique_ptr<EngineBase> create_engine_{d}_{n}_{vf}_{sf}_{hg}_{ns}();")
    lines.append("std::unique_ptr<EngineBase> make_engine(int ndims, int n, int vf, int sf, bool hg,"
                 " bool ns) {")
    lines.append("  const int h = hg ? 1 : 0, v = ns ? 1 : 0;")
    for (d, n, vf, sf, hg, ns) in cs:
        lines.append(f"  if (ndims == {d} && n == {n} && vf == {vf} && sf == {sf} && h == {hg}"
                     f" && v == {ns}) return create_engine_{d}_{n}_{vf}_{sf}_{hg}_{ns}();")
    lines.append("  return nullptr;")
    lines.append("}")
    lines.append("}  // namespace dgsem")
    _write_if_changed(path, "\n".join(lines) + "\n")
    files.append(path)
    return files


def _write_if_changed(path: str, text: str) -> None:
    if os.path.exists(path):
        with open(path) as f:
            if f.read() == text:
                return
    with open(path, "w") as f:
        f.write(text)


if __name__ == "__main__":
    for p in generate():
        print(p)
