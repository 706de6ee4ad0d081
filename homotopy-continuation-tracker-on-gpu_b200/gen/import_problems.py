"""Import problem folders from a GPU-HC checkout into this package.

For each selected problem, copies the reference-format folder
(gpuhc_settings.yaml, start_params.txt, target_params.txt, start_sols.txt,
dHdx_indx.txt, dHdt_indx.txt) into ``problems/<p>/`` and, for P2C problems,
derives ``p2c_terms.txt`` from the problem's ``sys_<p>.m`` with p2c_gen.derive
(which also checks both shipped tables against the polynomial system).

usage: python import_problems.py <GPU-HC-checkout-root> [problem ...]
(the root may also come from the GHC_REFERENCE_ROOT environment variable).
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import p2c_gen  # noqa: E402

PKG = os.path.dirname(HERE)
DEST = os.path.join(PKG, "problems")

DEFAULT_PROBLEMS = [
    "P3P",
    "5pt_rel_pos_alg_form_quat",
    "generalized_3views_4pts",
    "uncalibrated_trifocal_rel_pos_CY",
    "trifocal_2op1p_30x30",
    "3view_triangulation",
    "6pt_RS_abs_pos",
    "dual_reciever_TDOA_5pt",
    "distorted_2view_triangulation",
    "P3P_10x10",
    "3pt_rel_pos_homog",
    "4view_triangulation",
    "5pt_rel_pos_full_form_quat",
    "5pt_rel_pos_geo_form_quat",
    "6pt_RS_abs_pos_1lin",
    "PnP_unkn_principal_pt",
    "generalized_3views_6lines",
    "optimal_P4P_abs_pos",
    "optimal_PnP_quat",
    "rel_pos_quiver",
    "uncalibrated_trifocal_rel_pos_CH",
]

FILES = ["gpuhc_settings.yaml", "start_params.txt", "target_params.txt", "start_sols.txt",
         "dHdx_indx.txt", "dHdt_indx.txt"]

# problems whose system file name differs from the folder name
SYS_NAME = {"5pt_rel_pos_full_form_quat": "sys_5pt_rel_pos_full_form.m"}


def import_problem(root, name):
    src = os.path.join(root, "GPU-HC", "problems", name)
    dst = os.path.join(DEST, name)
    os.makedirs(dst, exist_ok=True)
    for f in FILES:
        shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
    y = p2c_gen.read_yaml_flat(os.path.join(dst, "gpuhc_settings.yaml"))
    if y.get("GPUHC_Type") == "P2C":
        sys_m = os.path.join(root, "auto-data-gen-tools", "p2c-problems",
                             SYS_NAME.get(name, "sys_%s.m" % name))
        info = p2c_gen.derive(dst, sys_m)
        p2c_gen.write_p2c_terms(os.path.join(dst, "p2c_terms.txt"), info, os.path.basename(sys_m))
        return "P2C M=%d K=%d" % (info["M"], info["K"])
    return y.get("GPUHC_Type")


def main(argv):
    root = argv[1] if len(argv) > 1 else os.environ.get("GHC_REFERENCE_ROOT")
    if not root:
        sys.exit(__doc__)
    names = argv[2:] or DEFAULT_PROBLEMS
    for n in names:
        try:
            print("%-36s %s" % (n, import_problem(root, n)))
        except Exception as e:  # report and continue with the others
            print("%-36s FAILED: %s" % (n, e))


if __name__ == "__main__":
    main(sys.argv)
