"""The C host shim (include/i2g_shim.c) compiles against include/i2g.h.

The shim replaces movemark()/ronurecalc() inside the reference build and reads
the reference's globals; here those globals are declared extern with the
reference's types (headmart.c:87-139, 175-279, 390-403), so the check needs
neither the reference sources nor a GPU.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

GLOBALS = r"""
#define MAXMRK 64000000
#define MAXTMR 200
extern long int xnumx, ynumy, nodenum, marknum;
extern double xsize, ysize, tmp_ambient, timestep, timesum, nubeg, nuend, nucontr;
extern int intermod, intermod1, outgrid, densimod, markmod, gridmod, viscmod, dynamo;
extern double M_acc, M_init, core_form_time, k_cutoff, relax_time, por_init, al2627_init, fe6056_init;
extern double gx[], gy[], vx[], vy[], pr[], exx[], eyy[], exy[], sxx[], syy[], sxy[], ga[], mu[];
extern double ro[], nu[], nd[], et[], cp[], kt[], ht[], tk[], po[], tk2[], tk3[], eps[], heatdif;
extern float markx[], marky[], markk[], markv[], markp[], markhi[], marktmax[], markpor[], markgr[], markacc[];
extern char markt[], markmg_old[];
extern double markmg_time[];
extern double marknu[MAXTMR], markdh[MAXTMR], markdv[MAXTMR], markss[MAXTMR], markmm[MAXTMR];
extern double markll[MAXTMR], marka0[MAXTMR], marka1[MAXTMR], markb0[MAXTMR], markb1[MAXTMR];
extern double marke0[MAXTMR], marke1[MAXTMR], markro[MAXTMR], markaa[MAXTMR], markbb[MAXTMR];
extern double markcp[MAXTMR], markkt[MAXTMR], markht[MAXTMR], markkf[MAXTMR], markkp[MAXTMR];
extern double markn0[MAXTMR], markn1[MAXTMR], marks0[MAXTMR], marks1[MAXTMR];
extern int markim[MAXTMR];
extern double td[350][350][2][5], tkmin, pbmin, tkstp, pbstp;
extern int tknum, pbnum, si_melting, fe_melting, ice_melting;
void tkrecalc();
"""


def shim_source():
    return open(os.path.join(ROOT, "include", "i2g_shim.c")).read()


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
@pytest.mark.parametrize("flags", [[], ["-DI2G_SHIM_RESIDENT"], ["-DI2G_SHIM_PRECISION=I2G_PREC_FP64"]],
                         ids=["default", "resident", "fp64"])
def test_shim_compiles(tmp_path, flags):
    src = tmp_path / "i2g_shim.c"
    src.write_text(GLOBALS + shim_source())
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-DUSE_I2G", *flags, "-I", os.path.join(ROOT, "include"),
                        "-c", str(src), "-o", str(tmp_path / "i2g_shim.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
