"""Builds the reference's own compute shaders as C++ into oracle/_ref/ (test
infrastructure: the oracle's cross-check against the reference itself).

The reference's full-search matcher runs on the GPU as GLSL compute shaders
(shaders/*.comp, dispatched by lib/nx_stereo/vulkan.ex:pipeline/1); there is
no Vulkan here, but the shader sources are C-like. This recipe reads them
where they lie under the reference checkout, rewrites their GLSL-only
declarations mechanically (buffer blocks into pointers the host binds,
specialisation constants into variables, `shared` arrays into statics,
`inout`/`out` parameters into references, `.xy` swizzles into calls, float
literals into f32 literals) and compiles every variant the reference
compiles (vulkan.ex @variants: the source plus its -D macros) against
glsl_cpu.h, whose fiber scheduler gives barrier() and the subgroup shuffles
their GLSL meaning. ref_pipeline.cpp dispatches the variants in the order
and with the workgroup counts, buffers and constants of vulkan.ex. Nothing
of the reference is copied into the repository: the rewritten sources and
the library exist only under oracle/_ref/ (git-ignored).

Run here, where the reference checkout exists; the built library travels
with the repository snapshot like the other built libraries.
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SRC = os.path.join(OUT, "src")
LIBRARY = os.path.join(OUT, "libnxs_ref_shaders.so")
REFERENCE = os.environ.get("NXS_REFERENCE", "/root/reference")
SHADERS = os.path.join(REFERENCE, "shaders")

# The matcher's variants (lib/nx_stereo/vulkan.ex:12-61): name -> (source, macros).
MATCHER = {
    "census": ("census_pair", []),
    "consistency": ("consistency_projected", []),
    "median": ("filter", []),
    "cost_horizontal_d128": ("cost_first", ["DISPARITIES=128", "FUSED=1"]),
}
BY_DISPARITIES = {
    "cost_forward": ("cost_first", []),
    "cost_reverse": ("cost_scan", ["PAIRED=1"]),
    "cost_down": ("cost_line", ["STEP_X=0", "STEP_Y=1"]),
    "cost_up": ("cost_line", ["STEP_X=0", "STEP_Y=-1"]),
    "cost_down_select": ("cost_line", ["STEP_X=0", "STEP_Y=1", "SELECT=1"]),
    "cost_down_right": ("cost_line", ["STEP_X=1", "STEP_Y=1", "PAIRED=1"]),
    "cost_down_left": ("cost_line", ["STEP_X=-1", "STEP_Y=1"]),
    "cost_up_right": ("cost_line", ["STEP_X=1", "STEP_Y=-1", "PAIRED=1"]),
    "cost_up_left": ("cost_line", ["STEP_X=-1", "STEP_Y=-1", "PAIRED=1"]),
    "select_8": ("select", []),
}
for _d in (64, 128):
    for _name, (_source, _macros) in BY_DISPARITIES.items():
        MATCHER[f"{_name}_d{_d}"] = (_source, [f"DISPARITIES={_d}"] + _macros)

# The stages' variants (lib/nx_stereo/kernels.ex:19-33) that the segment's
# stages around the matcher run on a GPU: name -> (source, macros).
STAGES = {
    "rectify_bytes": ("rectify", ["WORDS=0"]),
    "despeckle": ("despeckle", ["RADIUS=3"]),
    "temporal_filter": ("temporal_filter", ["MAX_MISSED=255"]),
    "depth": ("depth", []),
    "point_cloud_rows": ("point_cloud_rows", []),
    "disparity_rows": ("disparity_rows", []),
    "column_sums": ("column_sums", []),
}

# The coarse-to-fine search's variants (vulkan.ex:12-77): the shrink and
# band bases, the dense census windows, and per band width the band's costs,
# their column-major copy, the scans (a thread a line for bands 8 and 16,
# band_scan_lanes' lane groups for 32 and 64, whose 8-path form accumulates
# opposite pairs in band_scan_aggregate) and the selection.
COARSE_TO_FINE = {
    "shrink": ("shrink", []),
    "band_base": ("band_base", []),
    "census_dense": ("census_dense_pair", []),
    "census_blend": ("census_dense_pair", ["BLEND=1"]),
}
BY_BAND = {
    "band_cost": ("band_cost", []),
    "band_transpose_costs": ("band_transpose", []),
    "band_scan_horizontal": ("band_scan", ["DX=1", "DY=0"]),
    "band_scan_down": ("band_scan", ["DX=0", "DY=1"]),
    "band_select": ("band_select", ["PATHS=3"]),
    "band_select_8": ("band_select", ["PATHS=8"]),
}
NARROW_SCANS = {
    "band_scan_down_up": ("band_scan", ["DX=0", "DY=1", "DX2=0", "DY2=-1"]),
    "band_scan_down_diagonals": ("band_scan", ["DX=1", "DY=1", "DX2=-1", "DY2=1"]),
    "band_scan_up_diagonals": ("band_scan", ["DX=1", "DY=-1", "DX2=-1", "DY2=-1"]),
}
WIDE_SCANS = {
    "band_aggregate_vertical": ("band_scan_aggregate", ["DX=0", "DY=1", "FIRST=1"]),
    "band_aggregate_diagonal": ("band_scan_aggregate", ["DX=1", "DY=1"]),
    "band_aggregate_antidiagonal": ("band_scan_aggregate", ["DX=-1", "DY=1"]),
}
for _band in (8, 16, 32, 64):
    for _name, (_source, _macros) in {**BY_BAND, **(WIDE_SCANS if _band >= 32 else NARROW_SCANS)}.items():
        if _source == "band_scan" and _band >= 32:
            _source = "band_scan_lanes"
        if _name == "band_select_8" and _band >= 32:
            _macros = ["AGGREGATED=1"] + _macros
        COARSE_TO_FINE[f"{_name}_b{_band}"] = (_source, [f"BAND={_band}"] + _macros)

VARIANTS = dict(MATCHER)
VARIANTS.update(STAGES)
VARIANTS.update(COARSE_TO_FINE)

_COMMENTS = re.compile(r"//[^\n]*|/\*.*?\*/", re.S)
_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"\s*$', re.M)
_LOCAL_SIZE = re.compile(
    r"layout\s*\(\s*local_size_x\s*=\s*([^,)]+)(?:,\s*local_size_y\s*=\s*([^,)]+))?\s*\)\s*in\s*;")
_SPEC = re.compile(
    r"layout\s*\(\s*constant_id\s*=\s*(\d+)\s*\)\s*const\s+(int|float)\s+(\w+)\s*=\s*([^;]+);")
_BUFFER = re.compile(
    r"layout\s*\(\s*(?:set\s*=\s*\d+\s*,\s*)?binding\s*=\s*([\d\s+*()-]+?)\s*\)\s*((?:\w+\s+)*?)buffer\s+\w+\s*"
    r"\{\s*(\w+)\s+(\w+)\s*\[\s*[^\]]*\]\s*;\s*\}\s*;")
_ARRAY_CONSTRUCTOR = re.compile(r"\b(\w+)\s*\[\s*\w*\s*\]\s*\(")
_SHARED = re.compile(r"^\s*shared\s+(\w+)\s+(\w+)\s*((?:\[[^\]]+\]\s*)+);", re.M)
_FLOAT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+)(?![\w.])")
_SWIZZLE = re.compile(r"\.(xy|zw|xyz|xz|yz)\b(?!\s*\()")


def _read(name):
    with open(os.path.join(SHADERS, name)) as f:
        return f.read()


def _inline(name, seen):
    """The source with comments removed and its includes spliced in."""
    text = _COMMENTS.sub(" ", _read(name))

    def splice(m):
        inner = m.group(1)
        if inner in seen:  # the shaders include each file once
            return ""
        seen.add(inner)
        return _inline(inner, seen)

    return _INCLUDE.sub(splice, text)


def _parameters(text):
    """GLSL parameter qualifiers: inout/out become references (arrays decay
    to pointers, which GLSL's copy-in/copy-out matches for the arrays these
    shaders pass: none is written through a parameter without inout/out)."""
    text = re.sub(r"\b(?:inout|out)\s+(\w+)\s+(\w+)\s*\[", r"\1 \2[", text)
    text = re.sub(r"\b(?:inout|out)\s+(\w+)\s+(\w+)\b", r"\1 &\2", text)
    text = re.sub(r"([(,]\s*)in\s+(\w+\s+\w+)", r"\1\2", text)
    return text


def _array_constructors(text):
    """GLSL array constructors, T[N](a, b, ...), become brace lists {a, b, ...}
    (the shaders use them only to initialise a declared array)."""
    out, at = [], 0
    for m in _ARRAY_CONSTRUCTOR.finditer(text):
        if m.start() < at or m.group(1) not in ("uint", "int", "float", "uvec2", "uvec4", "vec2",
                                                 "vec4", "bool"):
            continue
        depth, i = 1, m.end()
        while depth:
            depth += {"(": 1, ")": -1}.get(text[i], 0)
            i += 1
        out.append(text[at:m.start()] + "{" + text[m.end():i - 1] + "}")
        at = i
    out.append(text[at:])
    return "".join(out)


def translate(source, macros):
    """C++ for one shader variant (its source preprocessed with its macros,
    as glslang does); returns (text, module facts)."""
    text = _inline(source + ".comp", set())
    lines = [ln for ln in text.splitlines() if not re.match(r"\s*#\s*(version|extension)\b", ln)]
    text = subprocess.run(["cpp", "-P", "-undef", *["-D" + m for m in macros], "-"],
                          input="\n".join(lines), capture_output=True, text=True, check=True).stdout
    facts = {"local_size": None, "spec": [], "bindings": [], "shared": []}

    def local_size(m):
        facts["local_size"] = m.group(1).strip()
        return "static const int nxs_local_size_x = (%s), nxs_local_size_y = (%s);" % (
            m.group(1).strip(), (m.group(2) or "1").strip())

    def spec(m):
        facts["spec"].append((int(m.group(1)), m.group(3), m.group(2) == "float"))
        return "%s %s = %s;" % (m.group(2), m.group(3), m.group(4).strip())

    def buffer(m):
        # a binding may be a constant expression of the preprocessed source (4 + 1)
        binding = m.group(1)
        if not re.fullmatch(r"[\d\s+*()-]+", binding):
            raise RuntimeError("binding " + binding)
        facts["bindings"].append((int(eval(binding, {"__builtins__": {}})), m.group(4)))
        return "%s *%s = nullptr;" % (m.group(3), m.group(4))

    def shared(m):
        dims = re.findall(r"\[([^\]]+)\]", m.group(3))
        if all(re.fullmatch(r"\s*\d+\s*", d) for d in dims):  # sizes fixed by the source
            return "static %s %s%s;" % (m.group(1), m.group(2), m.group(3))
        if len(dims) != 1:
            raise RuntimeError("a shared array of several dimensions sized at run time")
        facts["shared"].append((m.group(1), m.group(2), dims[0].strip()))
        return "NXS_SHARED(%s, %s, %s)" % (m.group(1), m.group(2), dims[0].strip())

    text = _LOCAL_SIZE.sub(local_size, text)
    text = _SPEC.sub(spec, text)
    text = _BUFFER.sub(buffer, text)
    text = _SHARED.sub(shared, text)
    text = _array_constructors(text)
    text = _parameters(text)
    text = _SWIZZLE.sub(r".\1()", text)
    text = _FLOAT.sub(lambda m: m.group(1) + "f", text)
    text = re.sub(r"\bvoid\s+main\s*\(", "void shader_main(", text)
    text = re.sub(r"\b(precise|highp|mediump|lowp|coherent|restrict)\b", "", text)
    if facts["local_size"] is None:
        raise RuntimeError(source + ": no local_size_x")
    return text, facts


def emit(name, source, macros):
    text, facts = translate(source, macros)
    ns = "v_" + name
    spec_ids = ", ".join(str(i) for i, _, _ in facts["spec"]) or "0"
    spec_ptrs = ", ".join("(void *)&%s::%s" % (ns, n) for _, n, _ in facts["spec"]) or "nullptr"
    spec_floats = ", ".join("1" if f else "0" for _, _, f in facts["spec"]) or "0"
    bind_ids = ", ".join(str(b) for b, _ in facts["bindings"]) or "0"
    bind_ptrs = ", ".join("(void **)&%s::%s" % (ns, n) for _, n in facts["bindings"]) or "nullptr"
    checks = "".join(
        "    if ((long long)(%s) > NXS_SHARED_CAP) return -1;\n    need += (long long)sizeof(%s) * (%s);\n"
        % (count, ty, count) for ty, _, count in facts["shared"])
    return f"""// Generated by oracle/build_ref.py from the reference's shaders/{source}.comp: do not edit.
#include "glsl_cpu.h"
namespace {ns} {{
{text}
static long long nxs_shared_bytes() {{
    long long need = 0;
{checks}    return need;
}}
}}  // namespace {ns}
extern "C" const nxs_module *nxs_module_{name}() {{
    static nxs_module m = {{"{name}", &{ns}::shader_main, {ns}::nxs_local_size_x,
        {ns}::nxs_local_size_y, {len(facts['spec'])}, {{{spec_ids}}}, {{{spec_ptrs}}},
        {{{spec_floats}}},
        {len(facts['bindings'])}, {{{bind_ids}}}, {{{bind_ptrs}}}, &{ns}::nxs_shared_bytes}};
    return &m;
}}
"""


def build(force=False, jobs=8):
    """Translates and compiles every variant; returns the library's path."""
    if not os.path.isdir(SHADERS):
        raise RuntimeError("the reference's shaders are not at " + SHADERS)
    os.makedirs(SRC, exist_ok=True)
    inputs = [os.path.join(HERE, f) for f in ("glsl_cpu.h", "glsl_runtime.cpp", "ref_pipeline.cpp",
                                               "build_ref.py")]
    inputs += [os.path.join(SHADERS, f) for f in os.listdir(SHADERS)]
    if not force and os.path.exists(LIBRARY):
        if os.path.getmtime(LIBRARY) >= max(os.path.getmtime(p) for p in inputs):
            return LIBRARY
    flags = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-I", HERE,
             "-Wno-unused-variable", "-Wno-unused-function"]
    objects, procs = [], []
    for name, (source, macros) in VARIANTS.items():
        cpp = os.path.join(SRC, name + ".cpp")
        with open(cpp, "w") as f:
            f.write(emit(name, source, macros))
        obj = os.path.join(SRC, name + ".o")
        objects.append(obj)
        procs.append(subprocess.Popen(["g++", *flags, "-c", cpp, "-o", obj]))
        if len(procs) >= jobs:
            if procs.pop(0).wait() != 0:
                raise RuntimeError("compiling a shader variant failed")
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("compiling a shader variant failed")
    declared = "".join('extern "C" const nxs_module *nxs_module_%s();\n' % n for n in VARIANTS)
    table = "".join('    {"%s", &nxs_module_%s},\n' % (n, n) for n in VARIANTS)
    modules = os.path.join(SRC, "modules.cpp")
    with open(modules, "w") as f:
        f.write('// Generated by oracle/build_ref.py: the table of shader variants.\n#include "glsl_cpu.h"\n'
                + declared + "struct nxs_module_entry { const char *name; const nxs_module *(*get)(); };\n"
                "extern const nxs_module_entry nxs_modules[] = {\n" + table + "    {nullptr, nullptr}};\n")
    command = ["g++", *flags, "-shared", "-o", LIBRARY + ".tmp", *objects, modules,
               os.path.join(HERE, "glsl_runtime.cpp"), os.path.join(HERE, "ref_pipeline.cpp")]
    subprocess.run(command, check=True)
    os.replace(LIBRARY + ".tmp", LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
