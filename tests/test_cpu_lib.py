"""libarc.so loads, exports the whole C ABI of include/arc_api.h, and its CPU scene generator
behaves (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np

from antiradiancecuts_b200 import _lib as L
from antiradiancecuts_b200 import scene

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(arc_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    declared = _declared_functions()
    assert len(declared) >= 25
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(L.SIGNATURES) <= declared


def test_struct_sizes():
    assert C.sizeof(L.ArcAvplHost) == 68
    assert C.sizeof(L.ArcMaterial) == 40
    assert C.sizeof(L.ArcBvhNode) == 36  # BvhNode (bvh.h:21-28)
    assert C.sizeof(L.ArcGBufferView) == 32


def test_status_strings_and_version():
    lib = L.load()
    assert lib.arc_api_version() == 1
    assert L.status_string(L.ARC_ERR_TOO_FEW_AVPLS) == "ARC_ERR_TOO_FEW_AVPLS"
    # every status the header declares has its own name
    hdr = open(os.path.join(ROOT, "include", "arc_api.h")).read()
    enum = re.search(r"typedef enum arc_status \{(.*?)\} arc_status;", hdr, re.S).group(1)
    declared = dict((n, int(v)) for n, v in re.findall(r"(ARC_\w+)\s*=\s*(\d+)", enum))
    assert len(declared) >= 10
    for name, value in declared.items():
        assert L.status_string(value) == name
    assert L.status_string(max(declared.values()) + 1) == "ARC_ERR_UNKNOWN"


def test_defaults():
    lib = L.load()
    p = L.ArcCutParams()
    lib.arc_cut_params_default(C.byref(p))
    assert abs(p.solid_angle_threshold - np.pi / 10) < 1e-6 and p.error_bound == np.float32(0.01)
    assert p.kind == L.ARC_CUT_ERROR_BOUND and p.ar_uncertain_factor == 16.0 and p.mlp_threshold == 0.5
    r = L.ArcRunConfig()
    lib.arc_run_config_default(C.byref(r))
    assert r.useLightCuts == 1 and abs(r.photonRadiusScale - 2.0) < 1e-7
    # CConfigManager's defaults: solid-angle cut at pi / 10, disk antiradiance, no clustered pass
    assert r.cut_kind == L.ARC_CUT_SOLID_ANGLE and abs(r.clusterRefinementThreshold - np.pi / 10) < 1e-6
    assert r.ar_kind == L.ARC_AR_DISK and r.useClusteredDeferred == 0 and r.precision == L.ARC_PREC_KAHAN
    assert abs(r.cluster_z_near - 0.1) < 1e-7 and abs(r.cluster_theta - np.radians(20.0)) < 1e-6
    g = L.ArcGatherParams()
    lib.arc_gather_params_default(C.byref(g))
    assert g.ar_kind == L.ARC_AR_CONE and abs(g.cone_half_angle - np.radians(30.0)) < 1e-6
    assert g.dist_clamp == 0.0 and g.precision == L.ARC_PREC_KAHAN and g.tile_config == -1
    b = L.ArcLbvhParams()
    lib.arc_lbvh_params_default(C.byref(b))
    assert b.bbox_mode == L.ARC_BBOX_SCENE and b.repr_seed == 5489 and b.consider_normals == 0 and b.wait_limit == 0


def test_null_arguments_are_rejected():
    lib = L.load()
    assert lib.arc_gather_bruteforce(None, None, None, L.f3(0, 0, 0), None, None) == L.ARC_ERR_INVALID_ARG
    assert lib.arc_context_create(0, None, None) == L.ARC_ERR_INVALID_ARG
    assert b"NULL" in lib.arc_last_error() or b"out" in lib.arc_last_error()


def test_every_entry_point_rejects_null_handles_before_any_cuda_call():
    """Every arc_status entry point of the header, called with NULL pointers and zero sizes, returns
    ARC_ERR_INVALID_ARG (the destroy functions accept NULL as a no-op) without touching CUDA (this
    machine has no GPU, so a CUDA call would have answered ARC_ERR_CUDA), and sets its own
    arc_last_error() message."""
    hdr = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "arc_api.h")).read(), flags=re.S)
    names = sorted(set(re.findall(r"\barc_status\s+(arc_[a-z0-9_]+)\s*\(", hdr)))
    assert len(names) >= 45
    lib = L.load()
    for name in names:
        _, argtypes = L.SIGNATURES[name]
        vals = []
        for a in argtypes:
            if isinstance(a, type) and issubclass(a, C.Structure):
                vals.append(a())
            elif a in (C.c_float, C.c_double):
                vals.append(0.0)
            elif a in (C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_size_t):
                vals.append(0)
            else:
                vals.append(None)
        lib.arc_context_create(0, None, None)  # leaves the message "out is NULL"
        marker = lib.arc_last_error()
        got = getattr(lib, name)(*vals)
        want = L.ARC_OK if name.endswith("_destroy") else L.ARC_ERR_INVALID_ARG
        assert got == want, (name, L.status_string(got), lib.arc_last_error())
        if got != L.ARC_OK and name != "arc_context_create":
            assert lib.arc_last_error() != marker, f"{name} failed without setting its own message"


def test_scene_generator_is_deterministic():
    d = scene.scene_desc(L.ARC_SCENE_ROOM_2BOXES, 2)
    a1, p1 = scene.trace_avpls(d, 2, 5000, 3)
    a2, p2 = scene.trace_avpls(d, 2, 5000, 3)
    assert p1 == p2 and a1.tobytes() == a2.tobytes()
    a3, _ = scene.trace_avpls(d, 3, 5000, 3)
    assert a1.tobytes() != a3.tobytes()


def test_avpl_semantics():
    # AvplShooter::createPath (AvplShooter.h:77-142): bounce >= 1, placed EPS behind the surface,
    # A = 0 on bounce 1 (explicit direct illumination), Russian roulette zeroes L with p = 0.2
    d = scene.scene_desc(L.ARC_SCENE_ROOM, 1)
    a, paths = scene.trace_avpls(d, 1, 20000, 3)
    assert (a["bounce"] >= 1).all() and (a["bounce"] <= 3).all()
    assert np.all(a["antiradiance"][a["bounce"] == 1] == 0)
    assert np.any(a["antiradiance"][a["bounce"] == 2] != 0)
    n = a["normal"]
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0)
    zero_L = np.all(a["incRadiance"] == 0, axis=1)
    not_last = a["bounce"] < 3
    frac = zero_L[not_last].mean()
    assert 0.1 < frac < 0.3
    w = a["incDirection"]
    assert np.allclose(np.linalg.norm(w, axis=1), 1.0, atol=1e-5)
    assert paths < 20000


def test_gbuffer_centre_pixel_hits_back_wall():
    d = scene.scene_desc(L.ARC_SCENE_ROOM, 1)
    pos, nrm = scene.gbuffer(d, 65, 65)
    c = (32, 32)
    assert abs(pos[c][2] - 1.0) < 1e-6 and nrm[c][3] == 1.0
    assert np.allclose(nrm[c][:3], [0, 0, -1])
    assert (nrm[..., 3] == 0).any()  # the corners see past the open front


def test_ctypes_layouts_match_the_header(tmp_path):
    """Every ctypes structure of _lib.py has the size and field offsets that the C compiler gives
    the header's struct of the same name (include/arc_api.h), so no call passes a skewed struct."""
    import inspect
    import os
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "arc_api.h")).read()
    structs = [(n, c) for n, c in inspect.getmembers(L, inspect.isclass)
               if issubclass(c, C.Structure) and f"typedef struct {n} " in header]
    assert len(structs) >= 15
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "arc_api.h"', "int main(void) {"]
    for n, c in structs:
        lines.append(f'    printf("{n} #sizeof %zu\\n", sizeof({n}));')
        for f in c._fields_:
            lines.append(f'    printf("{n} {f[0]} %zu\\n", offsetof({n}, {f[0]}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layouts.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layouts"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        n, field, v = line.split()
        got[(n, field)] = int(v)
    for n, c in structs:
        assert got[(n, "#sizeof")] == C.sizeof(c), n
        for f in c._fields_:
            assert got[(n, f[0])] == getattr(c, f[0]).offset, (n, f[0])


def test_plain_c_host_links_and_calls_the_library(tmp_path):
    """A C host (the reference's side of the boundary) compiles against include/arc_api.h, links
    libarc.so and calls it: host-only entry points, and an export written from C and read back."""
    import os
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "antiradiancecuts_b200")
    out_file = tmp_path / "c.pfm"
    src = tmp_path / "host.c"
    src.write_text(r"""
#include <stdio.h>
#include <string.h>
#include "arc_api.h"
int main(int argc, char** argv) {
    ArcRunConfig cfg;
    arc_run_config_default(&cfg);
    float px[2 * 2 * 4];
    for (int i = 0; i < 16; ++i) px[i] = (float)i;
    int s = arc_export_pfm(argv[1], px, 2, 2, 2);
    printf("%s %d %d %s\n", arc_status_string(s), cfg.useLightCuts, cfg.useClusteredDeferred,
           arc_status_string(ARC_ERR_INVALID_ARG));
    return s == ARC_OK ? 0 : 1;
}
""")
    exe = tmp_path / "host"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(root, "include"), str(src), "-L", libdir, "-larc",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(out_file)], check=True, capture_output=True, text=True)
    words = r.stdout.split()
    assert words[1:3] == ["1", "0"]
    assert out_file.read_bytes().startswith(b"PF\n2 2\n-1.0\n")


def test_cpp_host_compiles_warning_free_and_links(tmp_path):
    """The reference's host is C++: the header compiles as C++17 with every warning an error, its
    declarations have C linkage (the link resolves them in libarc.so), and a null context is
    rejected with ARC_ERR_INVALID_ARG before any CUDA call."""
    import os
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "antiradiancecuts_b200")
    src = tmp_path / "host.cpp"
    src.write_text(r"""
#include <cstdio>
#include <vector>
#include "arc_api.h"
int main() {
    ArcGatherParams gp;
    arc_gather_params_default(&gp);
    std::vector<ArcMaterial> mats(2);
    const arc_status s = arc_materials_upload(nullptr, mats.data(), (int32_t)mats.size());
    std::printf("%s %d %d\n", arc_status_string(s), gp.ar_kind, arc_mlp_num_params());
    return s == ARC_ERR_INVALID_ARG ? 0 : 1;
}
""")
    exe = tmp_path / "host"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(root, "include"), str(src),
                    "-L", libdir, "-larc", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], check=True, capture_output=True, text=True)
    assert r.stdout.split() == ["ARC_ERR_INVALID_ARG", str(L.ARC_AR_CONE), "9473"]
