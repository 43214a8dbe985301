"""Build the reference's own CUDA solver (RadChan src/montecarlo) for the B200.

Recipe (nothing from the reference is copied into this repository):
  1. copy the reference's solver sources from /root/reference into a temporary
     directory outside the repository;
  2. apply the minimal patches CUDA 12.9 and this GPU need
     - the legacy texture reference tex_Ib (removed in CUDA 12) becomes a
       texture object with the same clamp / linear-filter settings
       (mc_gpu_noint.cu:26, :787-791, and every tex2D(tex_Ib, ...));
     - the grey-gas table reader writes probg[nT][nB][nQ], one row past the end
       of a global array (read_tables.cpp:169-170); the patch writes
       probg[i][j][g] so no host memory outside the array is overwritten;
     - kernel_surface hands march_ray an Emission it never fills
       (mc_gpu_noint.cu:1330, "not going to be used since this is done only
       for adiabatic walls"); a wall bundle that reaches the opposite x wall
       when that wall is black and NOT adiabatic (the C2 case: adiabatic west
       wall, black east wall at 573 K) deposits Ibmax*tra*(invTi4*emiss.east
       - 1)*ratioI with emiss.east read from uninitialised memory
       (mc_gpu_noint.cu:432-440), which made the wall fluxes NaN.  The patch
       fills emiss from the wall spectra after the band draw exactly as
       kernel_fluid does (mc_gpu_noint.cu:157-175), through a __device__
       pointer to Ibw_d[gpu] set before the launch;
     - only in the "nb64s0fix" build: find_bandS's edge rule tests the wall
       CDF probs instead of the fluid CDF probd (mc_gpu_noint.cu:1189, :1208),
       the defect this solver does not reproduce, so that the wall fluxes of
       both solvers can be compared directly;
  3. rewrite the #define values of param.h (and the maxi/maxj/maxk initialisers)
     for the configuration; for the narrow-band configurations also nT/nQ/nB
     in NarrowBand.h and the constant g-CDF probq (mc_gpu_noint.cu:34-36,
     written for nQ = 16) as cumsum(wq) of the table set;
  4. compile with nvcc for sm_100a with the reference's own flags
     (--use_fast_math -ftz=true -prec-div=false, Makefile:20-24) together with
     oracle/ref_driver.cu into oracle/_ref/libref_<config>.so.

The library is a checker: tests/golden/make_ref_fixtures.py runs it on a B200
(one process per solve, because get_results_ calls cudaDeviceReset) and stores
its per-cell results as statistical parity fixtures.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF = os.environ.get("RADCHAN_REFERENCE", "/root/reference")
OUT = os.path.join(HERE, "_ref")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

MC_FILES = ["mc_gpu_noint.cu", "memory_copy_noint.cu", "read_tables.cpp", "definitions.h", "device_functions.h",
            "functions.h", "memory.h"]
PARAM_FILES = ["param.h", "NarrowBand.h"]

# Grey-gas channel, 32^3: kappa = 1/m, black walls at 955 K / 573 K, periodic
# y and z, photmax 64, nVar 4, one grid level.
CONFIGS = {
    "grey32": dict(defines=dict(num_gpu="1", p_col="1", imax="32", jmax="32", kmax="32", Lx="2.f",
                                Ly="6.283185307179586f", Lz="3.141592653589793f", fact_mesh="1.5", nVar="4",
                                photmax="64", chanHeight="1.0", grid_num="1", num_streams="2", blockdim="128",
                                nblocks="4096", srt="0", grey="1", calcwalls="0", random="0", floatpoint="0",
                                epsw="1.f", epse="1.f", epss="1.f", epsn="1.f", epsb="1.f", epst="1.f",
                                Tww="955", Twe="573", Tws="0", Twn="0", Twb="0", Twt="0", adiabw="0", adiabe="0",
                                toll="1.0e-3", tollS="1.0e-3", bdw="2", bde="2", bds="1", bdn="1", bdb="1", bdt="1"),
                   levels=["imax"], levels_j=["jmax"], levels_k=["kmax"]),
}

# Narrow-band channel, 64^3 (100 bands x 8 g points x 64 temperatures of the
# seeded synthetic tables), 3 levels 64/32/16 with maxs 5/5/1e5, photmax 256,
# nVar 4, wall-flux kernel with an adiabatic west wall; "nb64" with the
# band-sorted mode (srt = 1) as configured, "nb64s0" without it (its
# replicates are independent, so its sigma is a fair parity reference).
_NB = dict(num_gpu="1", p_col="1", imax="64", jmax="64", kmax="64", Lx="2.f", Ly="6.283185307179586f",
           Lz="3.141592653589793f", fact_mesh="1.5", nVar="4", photmax="256", chanHeight="1.0", grid_num="3",
           num_streams="2", blockdim="128", nblocks="4096", srt="1", grey="0", calcwalls="1", random="0",
           floatpoint="0", epsw="1.f", epse="1.f", epss="1.f", epsn="1.f", epsb="1.f", epst="1.f", Tww="955",
           Twe="573", Tws="0", Twn="0", Twb="0", Twt="0", adiabw="1", adiabe="0", toll="1.0e-3", tollS="1.0e-3",
           bdw="2", bde="2", bds="1", bdn="1", bdb="1", bdt="1")
for _name, _srt in (("nb64", "1"), ("nb64s0", "0"), ("nb64s0fix", "0")):
    CONFIGS[_name] = dict(defines=dict(_NB, srt=_srt), levels=["imax", "imax/2", "imax/4"],
                          levels_j=["jmax", "jmax/2", "jmax/4"], levels_k=["kmax", "kmax/2", "kmax/4"],
                          narrowband=dict(nT="64", nQ="8", nB="100"))
# "nb64s0fix" also corrects find_bandS's edge rule (see _patch_wall_edge), so
# that the wall fluxes can be compared with a solver that does not carry the
# defect; "nb64s0" keeps it.
CONFIGS["nb64s0fix"]["wall_edge_fix"] = True


def _patch_mc(src: str) -> str:
    old_decl = "texture<myfloat, cudaTextureType2D, cudaReadModeElementType> tex_Ib;"
    assert old_decl in src
    src = src.replace(old_decl, "__device__ cudaTextureObject_t rc_tex_Ib_obj;")
    src = src.replace("tex2D(tex_Ib,", "tex2D<myfloat>(rc_tex_Ib_obj,")
    bind = re.compile(r"tex_Ib\.addressMode\[0\].*?cudaBindTextureToArray\(tex_Ib, cuArrayI\[gpu\], DescIb\);", re.S)
    assert bind.search(src)
    src = bind.sub(
        "{ cudaResourceDesc rd; memset(&rd, 0, sizeof(rd)); rd.resType = cudaResourceTypeArray;\n"
        "  rd.res.array.array = cuArrayI[gpu];\n"
        "  cudaTextureDesc td; memset(&td, 0, sizeof(td));\n"
        "  td.addressMode[0] = cudaAddressModeClamp; td.addressMode[1] = cudaAddressModeClamp;\n"
        "  td.filterMode = cudaFilterModeLinear; td.readMode = cudaReadModeElementType; td.normalizedCoords = 0;\n"
        "  cudaTextureObject_t to; cudaCreateTextureObject(&to, &rd, &td, NULL);\n"
        "  cudaMemcpyToSymbol(rc_tex_Ib_obj, &to, sizeof(to)); }", src)
    if "#include <string.h>" not in src:
        src = "#include <string.h>\n" + src
    return _patch_surface_emission(src)


_SURF_FILL = """
#if adiabw == 0
					emiss.west  = rc_Ibw_ptr->west[nb];
#endif
#if adiabe == 0
					emiss.east  = rc_Ibw_ptr->east[nb];
#endif
#if bdt != 1
					emiss.top   = rc_Ibw_ptr->top[nb];
#endif
#if bdb != 1
					emiss.bot   = rc_Ibw_ptr->bot[nb];
#endif
#if bdn != 1
					emiss.north = rc_Ibw_ptr->north[nb];
#endif
#if bds != 1
					emiss.south = rc_Ibw_ptr->south[nb];
#endif
"""


def _patch_surface_emission(src: str) -> str:
    """kernel_surface: fill the Emission handed to march_ray from the wall
    spectra (mc_gpu_noint.cu:1330, :1418; kernel_fluid's rule :157-175)."""
    decl = "__device__ cudaTextureObject_t rc_tex_Ib_obj;"
    assert decl in src
    src = src.replace(decl, decl + "\n__device__ EmissSpec *rc_Ibw_ptr;", 1)
    k = src.index("__global__ void kernel_surface(")
    band = "\t\t\t\t\twvc  \t= wvc_d[nb];\n"
    j = src.index(band, k)
    src = src[:j + len(band)] + _SURF_FILL + src[j + len(band):]
    launch = "\t\t\tkernel_surface<<<"
    assert src.count(launch) == 1
    src = src.replace(launch, "\t\t\tcudaMemcpyToSymbol(rc_Ibw_ptr, &Ibw_d[gpu], sizeof(EmissSpec *));\n" + launch, 1)
    return src


def _patch_wall_edge(src: str) -> str:
    """find_bandS bisects the wall CDF probs but applies the R < cdf[0]
    edge rule to the fluid CDF probd (mc_gpu_noint.cu:1189, :1208): uniforms
    between probd[t][0] and probs[t][0] select band 1 instead of band 0.
    The patch tests probs[t-tm][0] in both branches."""
    k = src.index("__device__ __forceinline__ void find_bandS(")
    end = src.index("__device__ __forceinline__ void wave_find(", k)
    body = src[k:end]
    old = "if( Rwave <  probd[t-tm][0] )"
    old2 = "if(Rwave <  probd[t-tm][0] )"
    assert body.count(old) == 1 and body.count(old2) == 1
    body = body.replace(old, "if( Rwave <  probs[t-tm][0] )").replace(old2, "if(Rwave <  probs[t-tm][0] )")
    return src[:k] + body + src[end:]


def _patch_tables(src: str) -> str:
    old = re.compile(r"probg\[nT\]\[nB\]\[nQ\] = g;(\s*)probg_h\[m\] = probg\[nT\]\[nB\]\[nQ\];")
    assert old.search(src)
    return old.sub(r"probg[i][j][g] = g;\1probg_h[m] = probg[i][j][g];", src)


def _patch_probq(src: str, wq) -> str:
    """The 16-entry probq initializer (mc_gpu_noint.cu:34-36) becomes
    cumsum(wq) of the table set for other nQ."""
    pat = re.compile(r"(__device__ __constant__ myfloat probq\[nQ\] = \{)[^}]*(\};)", re.S)
    assert pat.search(src)
    c, vals = 0.0, []
    for w in wq:
        c += float(w)
        vals.append("%.9g" % c)
    vals[-1] = "1.0"
    return pat.sub(lambda m: m.group(1) + ",".join(vals) + m.group(2), src, count=1)


def _patch_narrowband(src: str, nb: dict) -> str:
    for k, v in nb.items():
        pat = re.compile(r"^(#define\s+%s\s+)(\S+)" % re.escape(k), re.M)
        assert pat.search(src), k
        src = pat.sub(lambda m: m.group(1) + v, src, count=1)
    return src


def _table_wq():
    sys.path.insert(0, ROOT)
    from radchan_b200 import workloads as W
    return list(W.tables_nb().arrays()["wq"])


def _patch_param(src: str, cfg: dict) -> str:
    for k, v in cfg["defines"].items():
        pat = re.compile(r"^(#define\s+%s\s+)(\S+)" % re.escape(k), re.M)
        assert pat.search(src), k
        src = pat.sub(lambda m: m.group(1) + v, src, count=1)
    for name, vals in (("maxi", cfg["levels"]), ("maxj", cfg["levels_j"]), ("maxk", cfg["levels_k"])):
        pat = re.compile(r"const int %s\[\] = \{[^}]*\};" % name)
        assert pat.search(src), name
        src = pat.sub("const int %s[] = {%s};" % (name, ", ".join(vals)), src, count=1)
    return src


def build(name: str, verbose: bool = False) -> str:
    cfg = CONFIGS[name]
    os.makedirs(OUT, exist_ok=True)
    lib = os.path.join(OUT, "libref_%s.so" % name)
    tmp = tempfile.mkdtemp(prefix="rc_refbuild_")
    try:
        mc = os.path.join(tmp, "src", "montecarlo")
        pa = os.path.join(tmp, "src", "param")
        os.makedirs(mc)
        os.makedirs(pa)
        for f in MC_FILES:
            shutil.copy(os.path.join(REF, "src", "montecarlo", f), mc)
        for f in PARAM_FILES:
            shutil.copy(os.path.join(REF, "src", "param", f), pa)
        patches = [(os.path.join(mc, "mc_gpu_noint.cu"), _patch_mc),
                   (os.path.join(mc, "read_tables.cpp"), _patch_tables),
                   (os.path.join(pa, "param.h"), lambda t: _patch_param(t, cfg))]
        if cfg.get("wall_edge_fix"):
            patches.append((os.path.join(mc, "mc_gpu_noint.cu"), _patch_wall_edge))
        if "narrowband" in cfg:
            wq = _table_wq()
            patches.append((os.path.join(mc, "mc_gpu_noint.cu"), lambda t: _patch_probq(t, wq)))
            patches.append((os.path.join(pa, "NarrowBand.h"), lambda t: _patch_narrowband(t, cfg["narrowband"])))
        for path, fn in patches:
            with open(path) as f:
                text = f.read()
            with open(path, "w") as f:
                f.write(fn(text))
        flags = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--use_fast_math", "-ftz=true",
                 "-prec-div=false", "-Xcompiler", "-fPIC", "-w"]
        objs = []
        for f in ("mc_gpu_noint.cu", "memory_copy_noint.cu", "read_tables.cpp"):
            o = os.path.join(tmp, f + ".o")
            cmd = [NVCC] + flags + ["-x", "cu" if f.endswith(".cu") else "c++", "-c", os.path.join(mc, f), "-o", o]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode:
                raise RuntimeError("reference build failed on %s:\n%s" % (f, r.stderr[-3000:]))
            objs.append(o)
        o = os.path.join(tmp, "ref_driver.o")
        r = subprocess.run([NVCC] + flags + ["-c", os.path.join(HERE, "ref_driver.cu"), "-o", o], capture_output=True,
                           text=True)
        if r.returncode:
            raise RuntimeError(r.stderr[-3000:])
        objs.append(o)
        r = subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib] + objs +
                           ["-L/usr/local/cuda/lib64", "-lcurand", "-Xlinker", "-rpath=/usr/local/cuda/lib64"], capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("reference link failed:\n" + r.stderr[-3000:])
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    if verbose:
        print(lib)
    return lib


def build_if_present() -> None:
    """Build every configuration when the reference sources are available."""
    if not os.path.isdir(os.path.join(REF, "src", "montecarlo")):
        return
    for name in CONFIGS:
        lib = os.path.join(OUT, "libref_%s.so" % name)
        newest = max(os.path.getmtime(__file__), os.path.getmtime(os.path.join(HERE, "ref_driver.cu")))
        if not os.path.exists(lib) or os.path.getmtime(lib) < newest:
            build(name)


if __name__ == "__main__":
    for n in (sys.argv[1:] or list(CONFIGS)):
        build(n, verbose=True)
