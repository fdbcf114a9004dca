"""Writes ntt_fam_*.cu: the kernel instantiations and their launchers.

    python csrc/gen_families.py      (from the package directory; the Makefile
                                      does not run it, the outputs are committed)

Every pass kernel is a template on (LOGR, LOGC): the tile is 2^LOGR rows by
2^LOGC columns with LOGR + LOGC = tile in {12, 13, 14} (make_plan_custom in
ntt_launch.cu only builds such plans), so its thread count, loop trip counts
and shared-memory offsets are compile-time constants. The launchers switch on
(logr, logc) and return cudaErrorInvalidConfiguration for anything else.
One file per family keeps the instantiations compiling in parallel.
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
TILES = (12, 13, 14)


def combos(rmax):
    return [(r, t - r) for t in TILES for r in range(6, min(rmax, t) + 1)]


COL = combos(12)   # first, middle and non-last inverse passes (radix <= 2^12)
ROW = combos(14)   # last forward / fused pass (radix <= 2^14)

FAMILIES = [
    ("ntt_fam_first.cu", "first forward pass (u32 limbs in)", "first", [
        ("k_fwd_first", COL, "launch_fwd_first",
         "(int logr, const PassGeo& g, cudaStream_t s, const u32* limbs, u64 ndig, u64* out, "
         "const RootTables& tw, const ProdJob* jobs, unsigned njobs, int operand)",
         "(limbs, ndig, out, g.logs, g.logm, tw, g.tfwd, jobs, operand)", "dim3(g.grid, njobs)")]),
    ("ntt_fam_mid.cu", "middle forward passes", "mid", [
        ("k_fwd_mid", COL, "launch_fwd_mid",
         "(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw, const ProdJob* jobs, "
         "unsigned njobs, int operand)",
         "(buf, g.logs, g.logm, tw, g.tfwd, jobs, operand, g.zstride)", "dim3(g.grid, njobs, g.zdim)")]),
    ("ntt_fam_inv.cu", "non-last inverse passes", "inv", [
        ("k_inv_mid", COL, "launch_inv_mid",
         "(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw, const ProdJob* jobs, "
         "unsigned njobs)",
         "(buf, g.logs, g.logm, tw, g.tinv, jobs, g.zstride)", "dim3(g.grid, njobs, g.zdim)")]),
    ("ntt_fam_last.cu", "last forward pass of operand A", "last", [
        ("k_fwd_last", ROW, "launch_fwd_last",
         "(int logr, const PassGeo& g, cudaStream_t s, u64* buf, const RootTables& tw, const ProdJob* jobs, "
         "unsigned njobs)",
         "(buf, tw, jobs, g.zstride)", "dim3(g.grid, njobs, g.zdim)")]),
    ("ntt_fam_fused.cu", "fused last pass of operand B (forward, pointwise, inverse)", "fused", [
        ("k_fused_last", ROW, "launch_fused_last",
         "(int logr, const PassGeo& g, cudaStream_t s, u64* bbuf, const u64* aspec, u64 ninv, "
         "const RootTables& tw, const ProdJob* jobs, unsigned njobs)",
         "(bbuf, aspec, ninv, tw, jobs, g.zstride)", "dim3(g.grid, njobs, g.zdim)")]),
]

SMALL = ("ntt_fam_small.cu", "single-CTA products, N <= 2^13", "small", "k_mul_small", range(2, 14),
         "launch_mul_small",
         "(int logn, const PassGeo& g, cudaStream_t s, const u32* a, u64 na, const u32* b, u64 nb, u32* out, "
         "u64 nout, unsigned long long* out_len, u64 ninv, const RootTables& tw, const ProdJob* jobs, "
         "unsigned njobs)",
         "(a, na, b, nb, out, nout, out_len, ninv, tw, jobs)", "dim3(g.grid * njobs)")

HEAD = ("// {fn} -- instantiations and launchers: {desc}.\n"
        "// Written by gen_families.py; kernel bodies are in ntt_kernels.cuh. With a\n"
        "// job table the grid's second dimension (the first, for single-CTA\n"
        "// products) runs over the jobs.\n"
        "#include \"ntt_kernels.cuh\"\n\nnamespace b2m {{\n")


def pass_family(fn, desc, tag, kerns):
    out = [HEAD.format(fn=fn, desc=desc)]
    cfg = []
    for kern, combs, launcher, sig, args, grid in kerns:
        out.append(f"\ncudaError_t {launcher}{sig} {{\n    switch (logr * 32 + g.logc) {{\n")
        for r, c in combs:
            out.append(f"        case {r * 32 + c}: {kern}<{r}, {c}><<<{grid}, g.block, g.smem, s>>>{args}; break;\n")
            cfg.append(f"    if (e == cudaSuccess) e = cudaFuncSetAttribute({kern}<{r}, {c}>, "
                       f"cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);\n")
        out.append("        default: return cudaErrorInvalidConfiguration;\n    }\n    return cudaGetLastError();\n}\n")
    out.append(f"\ncudaError_t configure_{tag}() {{\n    cudaError_t e = cudaSuccess;\n" + "".join(cfg)
               + "    return e;\n}\n\n}  // namespace b2m\n")
    return "".join(out)


def small_family():
    fn, desc, tag, kern, rng, launcher, sig, args, grid = SMALL
    out = [HEAD.format(fn=fn, desc=desc)]
    out.append(f"\ncudaError_t {launcher}{sig} {{\n    switch (logn) {{\n")
    cfg = []
    for n in rng:
        out.append(f"        case {n}: {kern}<{n}><<<{grid}, g.block, g.smem, s>>>{args}; break;\n")
        cfg.append(f"    if (e == cudaSuccess) e = cudaFuncSetAttribute({kern}<{n}>, "
                   f"cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);\n")
    out.append("        default: return cudaErrorInvalidConfiguration;\n    }\n    return cudaGetLastError();\n}\n")
    out.append(f"\ncudaError_t configure_{tag}() {{\n    cudaError_t e = cudaSuccess;\n" + "".join(cfg)
               + "    return e;\n}\n\n}  // namespace b2m\n")
    return "".join(out)


if __name__ == "__main__":
    for fn, desc, tag, kerns in FAMILIES:
        with open(os.path.join(HERE, fn), "w") as f:
            f.write(pass_family(fn, desc, tag, kerns))
    with open(os.path.join(HERE, SMALL[0]), "w") as f:
        f.write(small_family())
    print("wrote", ", ".join([x[0] for x in FAMILIES] + [SMALL[0]]))
