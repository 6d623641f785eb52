"""Regenerate tests/golden/ from the reference tree (run where it is mounted).

    python tests/golden/make_golden.py [/path/to/lammps-tensormd]

(default: TMD_REFERENCE_TREE, see oracle/reftree.py)

Copies five shipped potentials and two data files, and extracts the
published step-0 results of the reference (LAMMPS thermo lines and the
force.yaml dump, read as text) into published.json:

  examples/tensormd/binary/medium/output           96,000-atom MoNi_m3 run:
        step-0 energy (15 digits), pressure components, max force component
  examples/tensormd/binary/medium/force.yaml       per-atom step-0 forces
  examples/tensormd/trinary/a100_log/log_release.lammps     AlMgSi energy
  examples/tensormd/binary/medium/a100_log/log_release.lammps   MoNi_squareplus_500k
        step-0 energy and pressure (data file x 10x10x10, 100 K)
  examples/tensormd/W/tensormd/speedup/a100_log/log_0114.lammps  W_k32 energy
        and pressure (23,040 atoms)
  examples/tensormd/scaling/weak/200/log200.lammps   W_k32 step-0 energy and
        pressure of 200,000,000 BCC atoms
  examples/tensormd/W/tensormd/compare/a100_log/log{2,3,4,5}.lammps
        W_m3_k64_n128_squareplus step-0 energy and pressure of 46,080 to
        115,200 BCC atoms (log1, 23,040 atoms, is not used: its energy is
        1.46 eV and its pressure 876 bar away from the values the other four
        runs give per atom)

The test suite reads only the files written here.
"""
from __future__ import annotations

import json
import re
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main(ref: Path):
    ex = ref / "examples" / "tensormd"
    files = {
        "MoNi_m3.npz": ex / "binary/medium/MoNi_m3.npz",
        "MoNi_squareplus_500k.npz": ex / "binary/medium/MoNi_squareplus_500k.npz",
        "W_k32_snapshot.npz": ex / "W/tensormd/W_k32_snapshot.npz",
        "W_m3_k64_n128_squareplus.npz": ex / "W/tensormd/W_m3_k64_n128_squareplus.npz",
        "AlMgSi.24aug13.npz": ex / "trinary/AlMgSi.24aug13.npz",
        "Mo8_Ni8_id3210.data": ex / "binary/Mo8_Ni8_id3210.data",
        "AlMgSi.data": ex / "trinary/AlMgSi.data",
    }
    for dst, src in files.items():
        shutil.copyfile(src, HERE / dst)

    out = ex / "binary/medium/output"
    txt = out.read_text()
    m = re.search(r"Energy initial, next-to-last, final = \s*\n\s*(\S+)", txt)
    e96k = float(m.group(1))
    thermo0 = None
    for line in txt.splitlines():
        t = line.split()
        if len(t) == 8 and t[0] == "0":
            thermo0 = [float(v) for v in t]
            break
    fmax = float(re.search(r"Force max component initial, final = (\S+)", txt).group(1))
    forces = []
    for line in (ex / "binary/medium/force.yaml").read_text().splitlines():
        mm = re.match(r"\s*- \[\s*(\d+)\s*,\s*(\d+)\s*,\s*(\S+)\s*,\s*(\S+)\s*,\s*(\S+?)\s*,", line)
        if mm:
            forces.append([int(mm.group(1)), int(mm.group(2)), float(mm.group(3)),
                           float(mm.group(4)), float(mm.group(5))])

    def thermo_step0(path):
        """The step-0 thermo line as {column: value}."""
        header = None
        for line in path.read_text().splitlines():
            t = line.split()
            if t and t[0] == "Step":
                header = t
            elif header and t and t[0] == "0" and len(t) == len(header):
                return dict(zip(header, map(float, t)))
        raise RuntimeError(path)

    def thermo_pe(path):
        return thermo_step0(path)["PotEng"]

    def natoms(path):
        return int(re.search(r"Loop time of .* with (\d+) atoms", path.read_text()).group(1))

    wk64 = []
    for k in (2, 3, 4, 5):
        lg = ex / f"W/tensormd/compare/a100_log/log{k}.lammps"
        th = thermo_step0(lg)
        wk64.append({"natoms": natoms(lg), "pe": th["PotEng"], "press": th["Press"],
                     "volume": th["Volume"], "temp": th["Temp"]})

    almgsi = thermo_pe(ex / "trinary/a100_log/log_release.lammps")
    w_log = ex / "W/tensormd/speedup/a100_log/log_0114.lammps"
    w = thermo_pe(w_log)
    w_th = thermo_step0(w_log)
    sq_log = ex / "binary/medium/a100_log/log_release.lammps"
    sq = thermo_step0(sq_log)
    big_log = ex / "scaling/weak/200/log200.lammps"
    big = thermo_step0(big_log)
    pub = {
        "MoNi_m3": {
            "source": "examples/tensormd/binary/medium/output (data file x 10x20x30, "
                      "pair_coeff * * MoNi_m3.npz Mo Ni interp 0.0001, T = 0)",
            "replicas": 6000, "energy_total": e96k,
            "press": thermo0[4], "pxx": thermo0[5], "pyy": thermo0[6], "pzz": thermo0[7],
            "fmax_component": fmax, "interp": 1e-4, "elements": ["Mo", "Ni"],
        },
        "MoNi_m3_forces": {
            "source": "examples/tensormd/binary/medium/force.yaml (2x2x2 replica, "
                      "columns id type fx fy fz)",
            "rows": forces,
        },
        "AlMgSi": {
            "source": "examples/tensormd/trinary/a100_log/log_release.lammps "
                      "(AlMgSi.data x 10x10x3, interp 0.0001)",
            "replicas": 300, "energy_total": almgsi, "elements": ["Al", "Mg", "Si"],
            "interp": 1e-4,
        },
        "W_k32": {
            "source": "examples/tensormd/W/tensormd/speedup/a100_log/log_0114.lammps "
                      "(bcc 3.189, 24x24x20, interp 0.001)",
            "natoms": 23040, "energy_total": w, "lattice": 3.189, "interp": 1e-3,
            "elements": ["W"], "press": w_th["Press"], "volume": w_th["Volume"],
            "temp": w_th["Temp"],
        },
        "MoNi_squareplus": {
            "source": "examples/tensormd/binary/medium/a100_log/log_release.lammps "
                      "(data file x 10x10x10, pair_coeff * * MoNi_squareplus_500k.npz Mo Ni "
                      "interp 0.0001, step 0 of velocity create 100 K)",
            "replicas": 1000, "natoms": natoms(sq_log), "pe": sq["PotEng"],
            "press": sq["Press"], "temp": sq["Temp"], "interp": 1e-4, "elements": ["Mo", "Ni"],
        },
        "W_k32_200M": {
            "source": "examples/tensormd/scaling/weak/200/log200.lammps (bcc 3.189, "
                      "400x500x500, interp 0.001, step 0 of velocity create 300 K)",
            "natoms": natoms(big_log), "pe": big["PotEng"], "press": big["Press"],
            "volume": big["Volume"], "temp": big["Temp"],
        },
        "W_m3_k64": {
            "source": "examples/tensormd/W/tensormd/compare/a100_log/log2-5.lammps "
                      "(bcc 3.189, 24x24x40 to 24x24x100, interp 0.001, step 0 of "
                      "velocity create 300 K)",
            "runs": wk64, "lattice": 3.189, "interp": 1e-3, "elements": ["W"],
        },
    }
    (HERE / "published.json").write_text(json.dumps(pub, indent=1))
    print("wrote", HERE / "published.json")


if __name__ == "__main__":
    sys.path.insert(0, str(HERE.parent.parent / "oracle"))
    from reftree import reference_tree
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else reference_tree())
