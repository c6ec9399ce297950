"""Extract golden vectors from the reference's run protocol.

Reads dayfiles/wam_prot_coarse_ST6 of myWAveModel/WAM (the reference project,
path given as the first argument) and writes coarse_st6_protocol.json beside
this script.  The protocol is the only pinned output the reference ships; the
sections used here are the frequency/direction grid (:322-346), the DIA
index/weight tables printed by PRINT_SOURCE_STATUS (:876-936, written by
wam_source_module.f90:798-864), the depth/minimum-energy table parameters
(:942-957) and the CFL summary (:872-874).

Run in a container that holds the reference:
    python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import re
import sys


def floats(line):
    return [float(x) for x in re.findall(r"[-+]?\d*\.\d+(?:[EeDd][-+]?\d+)?|[-+]?\d+\.\d*(?:[EeDd][-+]?\d+)?", line)]


def main(ref):
    path = os.path.join(ref, "dayfiles", "wam_prot_coarse_ST6")
    lines = open(path, encoding="latin-1").read().splitlines()
    out = {"source": "dayfiles/wam_prot_coarse_ST6", "kl": 12, "ml": 25, "fr1": 0.04177248}

    def find(pat, start=0):
        for i in range(start, len(lines)):
            if pat in lines[i]:
                return i
        raise KeyError(pat)

    i = find("MODEL FREQUENCIES IN HERTZ")
    out["FR_5dp"] = floats(lines[i + 1]) + floats(lines[i + 2])
    i = find("MODEL DIRECTIONS IN DEGREE")
    out["TH_deg"] = floats(lines[i + 1])
    i = find("MODEL FREQUENCY INTERVALLS TIMES DIRECTION")
    out["DFIM_5dp"] = floats(lines[i + 1]) + floats(lines[i + 2])
    i = find("MODEL DEEP WATER GROUPVELOCITY")
    out["GOM_5dp"] = floats(lines[i + 1]) + floats(lines[i + 2])
    i = find("MODEL DEEP WATER PHASEVELOCITY")
    out["C_5dp"] = floats(lines[i + 1]) + floats(lines[i + 2])
    i = find("NUMBER OF PROPAGATION STEPS IN ONE CALL")
    out["NADV"] = int(lines[i].split("=")[-1])
    i = find("MAX. CFL NUMBER IS total_cfl")
    out["total_cfl"] = float(lines[i].split("=")[-1])
    i = find("ACL1       ACL2")
    vals = floats(lines[i + 1])
    out.update(dict(zip(["ACL1", "ACL2", "CL11", "CL21", "DAL1", "DAL2"], vals)))
    i = find("M   IKP IKP1  IKM IKM1")
    rows = []
    j = i + 1
    while lines[j].strip():
        t = lines[j].split()
        rows.append({"M": int(t[0]), "IKP": int(t[1]), "IKP1": int(t[2]), "IKM": int(t[3]), "IKM1": int(t[4]),
                     "FKLAP": float(t[5]), "FKLAP1": float(t[6]), "FKLAM": float(t[7]), "FKLAM1": float(t[8]),
                     "AF11": float(t[9])})
        j += 1
    out["dia_freq"] = rows
    i = find("K   K1W   K2W  K11W  K21W")
    ang = []
    for j in range(i + 1, i + 1 + 12):
        t = [int(x) for x in lines[j].split()]
        ang.append({"K": t[0], "K1W": [t[1], t[5]], "K2W": [t[2], t[6]], "K11W": [t[3], t[7]], "K21W": [t[4], t[8]]})
    out["dia_ang"] = ang
    i = find("TAIL ARRAY FRH")
    out["FRH"] = floats(lines[i + 1])
    i = find("DEPTH TABLE LENGTH")
    out["NDEPTH"] = int(lines[i].split(":")[-1])
    out["DEPTHD"] = float(lines[i + 1].split(":")[-1])
    out["DEPTHA"] = float(lines[i + 2].split(":")[-1])
    out["DEPTHE"] = float(lines[i + 3].split(":")[-1])
    i = find("WINDSPEED TABLE LENGTH")
    out["JUMAX"] = int(lines[i].split(":")[-1])
    out["DELU"] = float(lines[i + 1].split(":")[-1])
    out["UMAX"] = float(lines[i + 2].split(":")[-1])
    out["FETCH_MAX"] = float(lines[i + 3].split(":")[-1])
    out["FLMIN"] = float(lines[i + 4].split(":")[-1])
    i = find("PARAMETER FOR WIND INPUT ................ BETAMAX")
    out["BETAMAX"] = float(lines[i].split("=")[-1])
    out["CDFAC"] = float(lines[i + 1].split("=")[-1])
    out["ZALP"] = float(lines[i + 2].split("=")[-1])
    out["ALPHA"] = float(lines[i + 3].split("=")[-1])
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "coarse_st6_protocol.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the WAM Cycle 7 source tree>")
    main(sys.argv[1])
