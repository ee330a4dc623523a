"""The C-ABI library loads and exports every symbol include/lgh_b200.h
declares; host-only defaults match the reference (CPU, no compute call)."""

import ctypes
import os
import re
import subprocess

import pytest

import lgh_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "lgh_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(lgh_[a-z0-9_]+)\s*\(", src))
    return {n for n in names if not n.endswith("_fn")}


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(lgh_b200.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert _declared() <= set(lgh_b200.SIGNATURES), \
        sorted(_declared() - set(lgh_b200.SIGNATURES))


def test_defaults_match_reference():
    o = lgh_b200.glr_opts()           # glr_common_impl.h:295-312
    assert (o.ell, o.q_power, o.trunc_abs, o.trunc_rel, o.treat, o.seed,
            o.backend, o.nb, o.panel, o.grid2d, o.check) == \
        (200, 1, 0.0, 1e-3, 0, 271828, 0, 64, 64, 0, 1)
    p = lgh_b200.prior_opts()         # glr_common_impl.h:99-112
    assert (p.ksp_rtol, p.blocked_mode, p.tile, p.cheb_rtol, p.smax_krylov,
            p.smoother_top, p.nu_force, p.verbose) == \
        (1e-12, 0, 64, 1e-10, 1, 1.1, 0, 0)


def test_struct_layouts_match_c_compiler(tmp_path):
    """ctypes mirrors agree with gcc's layout of the header's structs."""
    structs = {"lgh_glr_opts_t": lgh_b200.GlrOpts,
               "lgh_glr_report_t": lgh_b200.GlrReport,
               "lgh_prior_mat_opts_t": lgh_b200.PriorMatOpts,
               "lgh_exec_opts_t": lgh_b200.ExecOpts,
               "lgh_glr_stats_t": lgh_b200.GlrStats,
               "lgh_prior_callbacks_t": lgh_b200.PriorCallbacks,
               "lgh_glr_correct_opts_t": lgh_b200.CorrectOpts,
               "lgh_glr_correct_report_t": lgh_b200.CorrectReport,
               "lgh_server_opts_t": lgh_b200.ServerOpts,
               "lgh_server_stats_t": lgh_b200.ServerStats,
               "lgh_comm_t": lgh_b200.Comm,
               "lgh_rows_comm_t": lgh_b200.RowsComm}
    lines = ['#include <stdio.h>', '#include <stddef.h>',
             '#include "lgh_b200.h"', 'int main(void){']
    for cname, py in structs.items():
        lines.append('printf("%%s %%zu\\n", "%s", sizeof(%s));'
                     % (cname, cname))
        for f, _ in py._fields_:
            lines.append('printf("%%s.%%s %%zu\\n", "%s", "%s", '
                         'offsetof(%s, %s));' % (cname, f, cname, f))
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"),
                           str(src), "-o", str(exe)])
    out = dict(l.rsplit(" ", 1) for l in
               subprocess.check_output([str(exe)]).decode().splitlines())
    for cname, py in structs.items():
        assert int(out[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(out[cname + "." + f]) == getattr(py, f).offset, \
                (cname, f)


def test_create_ksp_is_unsupported():
    L = lgh_b200.load()
    h = ctypes.c_void_p()
    rc = L.lgh_prior_create_ksp(None, None, None, ctypes.byref(h))
    assert rc == 56
    assert b"KSP" in L.lgh_last_error()
