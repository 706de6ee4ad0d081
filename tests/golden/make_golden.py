"""Copy the reference's checked-in golden run into tests/golden/.

GPU-HC/Output_Write_Files/GPU_Converged_HC_tracks.txt is one run of
uncalibrated_trifocal_rel_pos_CY at its shipped target parameters (444
converged endpoints of 12 unknowns, complex FP32).  It is stored here as
cy_golden_tracks.txt so the pin test does not need the reference tree.

usage: python make_golden.py [reference-root]
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GHC_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout> (or set GHC_REFERENCE_ROOT)")
    shutil.copyfile(os.path.join(root, "GPU-HC", "Output_Write_Files", "GPU_Converged_HC_tracks.txt"),
                    os.path.join(HERE, "cy_golden_tracks.txt"))
    print("wrote", os.path.join(HERE, "cy_golden_tracks.txt"))
