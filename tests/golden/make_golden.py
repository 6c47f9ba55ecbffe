"""Extracts the reference's frozen Stata fixtures into tests/golden/.

The reference (leoliu0/fereg) pins its OLS path against reghdfe 6.13.1 run at tol(1e-14)
(crates/fereg-core/tests/data/ols_data.csv + ols_s*.json, generated there by
gen_ols_fixtures.do). This script copies the data columns and the parts of each fixture the
tests here compare (b, V, dof_table, sample, resid, d, groupvar, scalars), and records each
fixture's model specification as restated from the reference's harness
(crates/fereg-core/tests/ols.rs:803-827).

It also extracts the IV fixtures (ivreghdfe 1.1.4 on an nlswork subset, iv_nls.csv +
iv_nls_{a,b}_{unadj,robust,cl1,cl2}_{none,aw,fw,pw}.json; harness tests/iv.rs:216-248) and the
logit fixtures (Stata `logit y x1 x2 i.fe1 i.fe2`, glm_logit.csv + glm_l_*.json; harness
tests/glm.rs:319-325, 659-672): b, V, sample and the scalars compared here; and the Poisson
fixtures (ppmlhdfe 2.3.3, glm_p_*.json on glm_gravity.csv, glm_auto.csv and glm_problem1.csv;
harness tests/glm.rs:432-480, 561-650) without separated observations.

Run once in a container that has the reference mounted:
    python tests/golden/make_golden.py /path/to/reference
The outputs are committed; the GPU box never reads the reference.
"""

import csv
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

IDYEAR = [["id"], ["year"]]
X3 = ["x1", "x2", "x3"]
X2 = ["x1", "x2"]


def fx(name, x, absorb, **kw):
    spec = dict(name=name, y="y", x=x, absorb=absorb, vce=[], robust=False, weight=None,
                weight_kind=None, singletons=True, noconstant=False, firstpair=False)
    spec.update(kw)
    return spec


# tests/ols.rs:803-827 (s16, with slopes, in SLOPE_SPECS below).
SPECS = [
    fx("s01_unadj", X3, IDYEAR),
    fx("s02_robust_3fe", X3, [["id"], ["year"], ["firm"]], robust=True),
    fx("s03_cluster_eq_fe", X2, IDYEAR, vce=["id"]),
    fx("s04_fe_nested_in_cluster", X3, IDYEAR, vce=["region"]),
    fx("s05_twoway_psd", X3, [["firm"], ["year"]], vce=["c1", "c2"]),
    fx("s06_aw_cluster", X3, IDYEAR, vce=["firm"], weight="w", weight_kind="aweight"),
    fx("s07_fw_robust", X3, IDYEAR, robust=True, weight="fw", weight_kind="fweight"),
    fx("s08_pw", X3, [["id"], ["year"], ["firm"]], weight="w", weight_kind="pweight"),
    fx("s09_absorbed_collinear", ["x1", "x2", "xa", "xc"], IDYEAR, status=[0, 0, 2, 3]),
    fx("s10_interaction", X2, [["id"], ["firm", "year"]]),
    fx("s11_noabsorb_cluster", X3, [], vce=["firm"]),
    fx("s12_noconstant", X2, IDYEAR, noconstant=True),
    fx("s13_keepsing_twoway", X2, IDYEAR, singletons=False, vce=["id", "year"]),
    fx("s14_groupvar", X2, [["id"], ["firm"], ["year"]]),
    fx("s15_firstpair_cluster", X2, [["id"], ["year"], ["firm"]], vce=["firm"], firstpair=True),
    fx("s17_y_absorbed", X2, IDYEAR, y="y2"),
    fx("s18_fw_twoway", X3, [["firm"], ["year"]], vce=["c1", "c2"], weight="fw", weight_kind="fweight"),
]

COLUMNS = ["id", "year", "firm", "region", "c1", "c2", "x1", "x2", "x3", "x4", "xa", "xc", "w", "fw", "y", "y2"]

# tests/ols.rs:827: reghdfe y x1 x2, absorb(id firm##c.x4), per term its intercept and slopes.
SLOPE_SPECS = [
    fx("s16_slopes", X2, [["id"], ["firm"]], intercept=[True, True], term_slopes=[[], ["x4"]]),
]


def main(ref):
    data_dir = os.path.join(ref, "crates", "fereg-core", "tests", "data")
    with open(os.path.join(data_dir, "ols_data.csv")) as f:
        rows = list(csv.DictReader(f))
    with open(os.path.join(HERE, "ols_data.csv"), "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(COLUMNS)
        for r in rows:
            w.writerow([r[c] for c in COLUMNS])
    out = []
    for spec in SPECS:
        with open(os.path.join(data_dir, f"ols_{spec['name']}.json")) as f:
            j = json.load(f)
        tag = spec["name"][1:3]
        fix = dict(spec=spec, cmdline=j["cmdline"], colnames=j["colnames"], b=j["b"], V=j["V"],
                   dof_table=j["dof_table"], sample=j["sample"], scalars=j["scalars"])
        for key in (f"r{tag}", f"d{tag}", f"gv{tag}"):
            if key in j:
                fix[key[: -2]] = j[key]
        out.append(fix)
    with open(os.path.join(HERE, "ols_fixtures.json"), "w") as f:
        json.dump(out, f)
    print(f"wrote {len(out)} fixtures, {len(rows)} rows")
    out = []
    for spec in SLOPE_SPECS:
        with open(os.path.join(data_dir, f"ols_{spec['name']}.json")) as f:
            j = json.load(f)
        out.append(dict(spec=spec, cmdline=j["cmdline"], colnames=j["colnames"], b=j["b"], V=j["V"],
                        dof_table=j["dof_table"], sample=j["sample"], scalars=j["scalars"]))
    with open(os.path.join(HERE, "ols_slopes_fixtures.json"), "w") as f:
        json.dump(out, f)
    print(f"wrote {len(out)} slope fixtures")


IV_COLUMNS = ["idcode", "year", "ln_wage", "age", "tenure", "union", "south", "msp", "w", "fw"]
IV_SCALARS = ["N", "df_r", "df_m", "df_a", "sdofminus", "rss", "rmse", "F", "N_clust", "endog_ct", "inexog_ct",
              "exexog_ct"]
LOGIT_COLUMNS = ["y", "y2", "x1", "x2", "fe1", "fe2", "c"]
# tests/glm.rs:659-672: unweighted logit fixtures with absorbed FE (fw / pw / noabsorb are outside
# the device path's scope)
LOGIT_SPECS = [
    dict(name="l_oim", absorb=["fe1", "fe2"], vce="oim", cluster=None),
    dict(name="l_robust", absorb=["fe1", "fe2"], vce="robust", cluster=None),
    dict(name="l_cluster", absorb=["fe1", "fe2"], vce="cluster", cluster="c"),
    dict(name="l_onefe", absorb=["fe1"], vce="oim", cluster=None),
]


def copy_csv(src, dst, columns):
    with open(src) as f:
        rows = list(csv.DictReader(f))
    with open(dst, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(columns)
        for r in rows:
            w.writerow([r[c] for c in columns])
    return len(rows)


def main_iv_logit(ref):
    data_dir = os.path.join(ref, "crates", "fereg-core", "tests", "data")
    copy_csv(os.path.join(data_dir, "iv_nls.csv"), os.path.join(HERE, "iv_nls.csv"), IV_COLUMNS)
    out = []
    for tag, inst in (("a", ["union", "south"]), ("b", ["union", "south", "msp"])):
        for v in ("unadj", "robust", "cl1", "cl2"):
            for wt in ("none", "aw", "fw", "pw"):
                name = f"nls_{tag}_{v}_{wt}"
                with open(os.path.join(data_dir, f"iv_{name}.json")) as f:
                    j = json.load(f)
                spec = dict(name=name, absorb=["idcode", "year"], y="ln_wage", exog=["age"], endog=["tenure"],
                            inst=inst, weight={"aw": "w", "pw": "w", "fw": "fw"}.get(wt),
                            weight_kind={"aw": "aweight", "pw": "pweight", "fw": "fweight"}.get(wt),
                            cluster={"cl1": ["idcode"], "cl2": ["idcode", "year"]}.get(v, []),
                            vce={"unadj": "unadjusted", "robust": "robust"}.get(v, "cluster"))
                sc = {k: j["scalars"].get(k) for k in IV_SCALARS}
                out.append(dict(spec=spec, cmdline=j["cmdline"], b=j["b"], V=j["V"], sample=j["sample"], scalars=sc))
    with open(os.path.join(HERE, "iv_fixtures.json"), "w") as f:
        json.dump(out, f)
    copy_csv(os.path.join(data_dir, "glm_logit.csv"), os.path.join(HERE, "glm_logit.csv"), LOGIT_COLUMNS)
    out = []
    for spec in LOGIT_SPECS:
        with open(os.path.join(data_dir, f"glm_{spec['name']}.json")) as f:
            j = json.load(f)
        p = len(j["b"])
        V = [j["V"][a * p + b] for a in range(2) for b in range(2)]
        sc = {k: j["scalars"][k] for k in ("N", "ll", "ll_0", "converged")}
        out.append(dict(spec=spec, cmdline=j["cmdline"], b=j["b"][:2], V=V, sample=j["sample"], scalars=sc))
    with open(os.path.join(HERE, "logit_fixtures.json"), "w") as f:
        json.dump(out, f)
    print("wrote the IV and logit fixtures")


# tests/glm.rs:561-650: ppmlhdfe 2.3.3 fixtures with no separated observation, unweighted and
# without offset (the scope of the device IRLS). Each spec restates the harness's: data set,
# outcome, regressors, absorbed terms (interactions as lists), cluster dimensions, vce, whether
# singletons are kept, the solver tolerance, and rows excluded before the call (`exclude`,
# 1-based observation numbers of the fixture's `if` condition).
POISSON_SPECS = [
    dict(name="p_gravity", data="gravity", y="trade", x=["rta", "x2"],
         absorb=[["exp", "year"], ["imp", "year"], ["exp", "imp"]], cluster=[["exp", "imp"]], vce="cluster",
         keepsing=False, tol=1e-10, exclude=[]),
    dict(name="p_twoway_robust", data="auto", y="price", x=["weight", "gear_ratio", "length"],
         absorb=[["turn"], ["trunk"]], cluster=[], vce="robust", keepsing=True, tol=1e-12, exclude=[]),
    # V not compared: ppmlhdfe's two-way cluster V is the eigenvalue-clipped bordered matrix with
    # _cons on its internal standardized scale (glm/mod.rs:1054-1120); this path reports no
    # _cons and clips the regressors' block. b, the sample, N and N_clust are compared.
    dict(name="p_twoway_cluster2", data="auto", y="price", x=["weight", "gear_ratio", "length"],
         absorb=[["turn"], ["trunk"]], cluster=[["turn"], ["trunk"]], vce="cluster", keepsing=True, tol=1e-12,
         exclude=[], compare_v=False),
    dict(name="p_twoway_cluster_turn", data="auto", y="price", x=["weight", "gear_ratio", "length"],
         absorb=[["turn"], ["trunk"]], cluster=[["turn"]], vce="cluster", keepsing=False, tol=1e-12, exclude=[]),
    dict(name="p_d_twoway", data="auto", y="price", x=["weight", "gear_ratio", "length"],
         absorb=[["turn"], ["trunk"]], cluster=[], vce="robust", keepsing=False, tol=1e-12, exclude=[]),
    dict(name="p_savefe", data="auto", y="price", x=["weight", "gear_ratio"], absorb=[["turn"], ["foreign"]],
         cluster=[], vce="robust", keepsing=True, tol=1e-10, exclude=[]),
    dict(name="p_guess_ols", data="auto", y="price", x=["weight", "gear_ratio", "length"], absorb=[["turn"]],
         cluster=[], vce="robust", keepsing=False, tol=1e-10, exclude=[]),
    dict(name="p_problem1", data="problem1", y="y", x=["x1", "x2"], absorb=[["i"], ["j"]], cluster=[],
         vce="robust", keepsing=False, tol=1e-10, exclude=[5, 7, 8, 14, 15]),
]
POISSON_DATA = {
    "gravity": ["trade", "rta", "x2", "exp", "imp", "year"],
    "auto": ["price", "weight", "gear_ratio", "length", "turn", "trunk", "foreign"],
    "problem1": ["y", "x1", "x2", "i", "j"],
}
POISSON_SCALARS = ["N", "num_separated", "num_singletons", "N_clust", "ll", "ll_0", "deviance", "chi2", "rank",
                   "df_m"]


# tests/glm.rs:549-590: ppmlhdfe 2.3.3 fixtures fitted with sep(fe relu) (the reference's
# Session::glm_separate rounds), unweighted and without offset. `first_obs`: rows before it are
# excluded (the fixture's `if _n > 2`); `counts`: the harness's (num_separated, num_singletons)
# where they differ from the fixture's (p_problem1: ppmlhdfe's own check gave up on the full
# data, so its fixture holds the sample its test expects).
SEP_SPECS = [
    dict(name="p_problem1", data="problem1", y="y", x=["x1", "x2"], absorb=[["i"], ["j"]], keepsing=False,
         tol=1e-10, first_obs=0, counts=[4, 1], maxiter=10000),
    dict(name="p_problem2", data="problem2", y="y", x=["x1", "x2"], absorb=[["i"], ["j"]], keepsing=False,
         tol=1e-10, first_obs=0, counts=None, maxiter=10000),
    dict(name="p_problem3", data="problem3", y="y", x=["x1", "x2", "x3"], absorb=[], keepsing=False, tol=1e-12,
         first_obs=0, counts=None, maxiter=10000),
    dict(name="p_problem4", data="problem4", y="y", x=["x1", "x2", "x3"], absorb=[], keepsing=False, tol=1e-12,
         first_obs=0, counts=None, maxiter=200),
    dict(name="p_problem5", data="problem5", y="y", x=["x1", "x2"], absorb=[["i"], ["j"]], keepsing=False,
         tol=1e-12, first_obs=0, counts=None, maxiter=10000),
    dict(name="p_problem6", data="problem6", y="y", x=["x"], absorb=[], keepsing=False, tol=1e-10, first_obs=0,
         counts=None, maxiter=10000),
    dict(name="p_hard1", data="hard1", y="y", x=[], absorb=[["id1"], ["id2"]], keepsing=False, tol=1e-10,
         first_obs=0, counts=None, maxiter=10000),
    dict(name="p_hard2_keepsing", data="hard2", y="FTA", x=[], absorb=[["ijk_fe"], ["jkt_fe"], ["ikt_fe"]],
         keepsing=True, tol=1e-12, first_obs=0, counts=None, maxiter=10000),
    dict(name="p_hard3", data="hard3", y="y", x=[], absorb=[["id1"], ["id2"]], keepsing=False, tol=1e-10,
         first_obs=0, counts=None, maxiter=10000),
    dict(name="p_hard5", data="hard5", y="y", x=["x1", "x2", "x3", "x4"], absorb=[], keepsing=False, tol=1e-10,
         first_obs=0, counts=None, maxiter=10000),
    dict(name="p_hard5b", data="hard5", y="y", x=["x2", "x3", "x4"], absorb=[], keepsing=False, tol=1e-10,
         first_obs=0, counts=None, maxiter=10000),
    dict(name="p_hard4", data="hard5", y="y", x=["x2", "x3", "x4"], absorb=[], keepsing=False, tol=1e-10,
         first_obs=2, counts=None, maxiter=10000),
]
SEP_DATA = {
    "problem1": ["y", "x1", "x2", "i", "j"],
    "problem2": ["y", "x1", "x2", "i", "j"],
    "problem3": ["y", "x1", "x2", "x3"],
    "problem4": ["y", "x1", "x2", "x3"],
    "problem5": ["y", "x1", "x2", "i", "j"],
    "problem6": ["y", "x"],
    "hard1": ["y", "id1", "id2"],
    "hard2": ["FTA", "ikt_fe", "jkt_fe", "ijk_fe"],
    "hard3": ["y", "id1", "id2"],
    "hard5": ["y", "x1", "x2", "x3", "x4", "x5"],
}


def main_separation(ref):
    data_dir = os.path.join(ref, "crates", "fereg-core", "tests", "data")
    for name, cols in SEP_DATA.items():
        copy_csv(os.path.join(data_dir, f"glm_{name}.csv"), os.path.join(HERE, f"glm_{name}.csv"), cols)
    out = []
    for spec in SEP_SPECS:
        with open(os.path.join(data_dir, f"glm_{spec['name']}.json")) as f:
            j = json.load(f)
        sc = {k: j["scalars"].get(k) for k in POISSON_SCALARS}
        out.append(dict(spec=spec, cmdline=j["cmdline"], colnames=j["colnames"], b=j["b"], V=j["V"],
                        sample=j["sample"], scalars=sc))
    with open(os.path.join(HERE, "separation_fixtures.json"), "w") as f:
        json.dump(out, f)
    print(f"wrote {len(out)} separation fixtures")


# tests/vce.rs:557-615: CRV3 fixtures of OLS on vce_cs.csv (do-file jackknife loops of reghdfe).
CRV3_SPECS = [
    dict(name="crv3_ols_nested", y="y", x=["x1", "x2"], absorb=["f1", "f2"], cluster=["c"], weight=None,
         weight_kind=None),
    dict(name="crv3_ols_aw", y="y", x=["x1", "x2"], absorb=["f1", "f2"], cluster=["c"], weight="w",
         weight_kind="aweight"),
    dict(name="crv3_ols_c2", y="y", x=["x1", "x2"], absorb=["f2"], cluster=["c2"], weight=None, weight_kind=None),
    dict(name="crv3_ols_twoway", y="y", x=["x1", "x2"], absorb=["f2"], cluster=["c", "c2"], weight=None,
         weight_kind=None),
]
VCE_CS_COLUMNS = ["f1", "f2", "c", "c2", "z1", "z2", "x1", "x2", "en", "y", "yp", "w", "fw"]


# tests/vce.rs:509-550: Stata 19 `regress y x1 x2 i.f1 i.f2, vce(hc2|hc3)` on vce_cs.csv (the x
# block compared with absorbed f1 f2; all of b and V without them).
HC_SPECS = [dict(name=f"{hc}_{wt}", hc=hc, absorb=(wt != "noabsorb"),
                 weight={"aw": "w", "pw": "w", "fw": "fw"}.get(wt),
                 weight_kind={"aw": "aweight", "pw": "pweight", "fw": "fweight"}.get(wt))
            for hc in ("hc2", "hc3") for wt in ("none", "aw", "fw", "noabsorb") + (("pw",) if hc == "hc2" else ())]


def main_hc(ref):
    data_dir = os.path.join(ref, "crates", "fereg-core", "tests", "data")
    out = []
    for spec in HC_SPECS:
        with open(os.path.join(data_dir, f"vce_{spec['name']}.json")) as f:
            j = json.load(f)
        sc = {k: j["scalars"].get(k) for k in ("N", "df_r")}
        out.append(dict(spec=spec, cmdline=j["cmdline"], b=j["b"], V=j["V"], sample=j["sample"], scalars=sc))
    with open(os.path.join(HERE, "hc_fixtures.json"), "w") as f:
        json.dump(out, f)
    print(f"wrote {len(out)} HC2 / HC3 fixtures")


def main_crv3(ref):
    data_dir = os.path.join(ref, "crates", "fereg-core", "tests", "data")
    copy_csv(os.path.join(data_dir, "vce_cs.csv"), os.path.join(HERE, "vce_cs.csv"), VCE_CS_COLUMNS)
    out = []
    for spec in CRV3_SPECS:
        with open(os.path.join(data_dir, f"vce_{spec['name']}.json")) as f:
            j = json.load(f)
        sc = {k: j["scalars"].get(k) for k in ("N", "N_clust", "df_r", "df_a", "num_singletons")}
        out.append(dict(spec=spec, cmdline=j["cmdline"], b=j["b"], V=j["V"], sample=j["sample"], scalars=sc))
    with open(os.path.join(HERE, "crv3_fixtures.json"), "w") as f:
        json.dump(out, f)
    print(f"wrote {len(out)} CRV3 fixtures")


def main_poisson(ref):
    data_dir = os.path.join(ref, "crates", "fereg-core", "tests", "data")
    for name, cols in POISSON_DATA.items():
        copy_csv(os.path.join(data_dir, f"glm_{name}.csv"), os.path.join(HERE, f"glm_{name}.csv"), cols)
    out = []
    for spec in POISSON_SPECS:
        with open(os.path.join(data_dir, f"glm_{spec['name']}.json")) as f:
            j = json.load(f)
        sc = {k: j["scalars"].get(k) for k in POISSON_SCALARS}
        out.append(dict(spec=spec, cmdline=j["cmdline"], colnames=j["colnames"], b=j["b"], V=j["V"],
                        sample=j["sample"], scalars=sc))
    with open(os.path.join(HERE, "poisson_fixtures.json"), "w") as f:
        json.dump(out, f)
    print(f"wrote {len(out)} Poisson fixtures")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    ref = sys.argv[1]
    main(ref)
    main_iv_logit(ref)
    main_poisson(ref)
    main_separation(ref)
    main_crv3(ref)
    main_hc(ref)
