"""The Python binding's ctypes structures against the C header: a small C
program compiled against include/mc_abi.h prints each structure's size and
field offsets, and the binding must agree field by field (a field added to
the header but not to the binding, or in another place, shifts every field
after it)."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

import mcpt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (C type, binding class, fields compared by name)
STRUCTS = [
    ("mc_guide_config", mcpt.GuideConfig,
     ["bounds", "learning_rate", "beta1", "beta2", "epsilon", "seed", "batch_capacity", "guide_fraction", "train_steps",
      "train_vertices", "direction_input", "guided_depth", "weight_cap", "fold_below", "anchor_lobes", "nee_records"]),
    ("mc_bvh_build_opts", mcpt.BvhBuildOpts, ["permutation", "layout", "keep_reference_nodes", "builder",
                                               "phase_launches"]),
    ("mc_render_params", mcpt.RenderParams,
     ["camera", "width", "height", "spp", "first_sample", "max_depth", "persistent", "rng", "seed", "intersector",
      "disable_clamp", "queue_capacity", "refill_threshold", "use_graph", "instrument", "samples_per_wave",
      "env_sampling", "stack_entries", "trace_threads"]),
    ("mc_render_stats", mcpt.RenderStats,
     ["extend_rays", "shadow_rays", "paths", "node_visits", "leaf_tests", "render_ms", "trace_ms", "trace_launches",
      "kernel_launches", "error_flags", "shade_ms", "guide_infer_ms", "guide_train_ms"]),
    ("mc_server_config", mcpt.ServerConfig, ["hbm_budget_bytes", "max_active", "samples_per_step", "wave_paths", "flags"]),
]


@pytest.fixture(scope="module")
def layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("abi")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "mc_abi.h"', "int main(void) {"]
    for ctype, _, fields in STRUCTS:
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (ctype, ctype))
        for f in fields:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (ctype, f, ctype, f))
    lines += ["return 0;", "}"]
    src = d / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "probe"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.split("\n"):
        if line:
            t, f, v = line.split()
            table[(t, f)] = int(v)
    return table


@pytest.mark.parametrize("ctype,cls,fields", STRUCTS, ids=[s[0] for s in STRUCTS])
def test_binding_matches_the_header(layout, ctype, cls, fields):
    assert C.sizeof(cls) == layout[(ctype, "size")]
    for f in fields:
        assert getattr(cls, f).offset == layout[(ctype, f)], f
