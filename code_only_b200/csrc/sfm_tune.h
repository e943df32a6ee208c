// sfm_tune.h -- the table of the autotuner (host code only).
//
// The solver's kernels come in launch-shape variants that differ only in how
// the work is spread over threads and CTAs; every variant evaluates the same
// expressions in the same order, so that choice never changes a result bit.
// A table maps (knob, element size, block edge, AMR level, fill kind) to the
// chosen variant; Solver::autotune fills it by timing the candidates on the
// context's own hierarchy, sfm_tune_save / sfm_tune_load keep it across
// runs.  Launch-shape knobs:
//   ghost_fill    level fill by the three directional passes (0) or by one
//                 launch per level (1; only where Solver::ghost_merge_ok);
//                 key: element size, block edge n, AMR level, fill kind
//   relax_threads threads of the bulk-copy smoother CTA (256, 288, 512 or
//                 544); key: element size, block edge n, kind -1 for the
//                 two colour launches, 1 for the fused sweep
//   resid_bpc     blocks per CTA of the tiled residual (1, 2 or 4);
//                 key: element size, block edge n
//   base_ctas     CTAs of the base-grid multigrid launch: 1, or a cluster
//                 of 2, 4, 8 or 16 (sfm_mg.cuh); key: element size, base
//                 grid cells per edge
//   base_wide     with a cluster, the smallest level (cells per edge: 16,
//                 32 or 64) whose steps use every CTA; same key
// and, for the mixed-precision path only (element size 4), the schedule of
// the FP32 inner solve, which is a preconditioner inside the FP64 defect
// correction: the outer loop converges to the same potential whatever the
// schedule, only its cost and the number of outer iterations change (the
// FP64 path always runs the reference's schedule):
//   fmg_ncycle      V-cycles per fmg level in fmg_lin (reference 2, fmg.F90:280-288)
//   fmg_sweeps      pre- and post-smoothing sweeps in fmg_lin (reference 2)
//   vmg_sweeps      pre- and post-smoothing sweeps in vmg_fas (reference 2, vmg.F90:125-135)
//   base_corrections  cap on mg_cycle's defect corrections (reference 10, mg.F90:50-52)
//   fused_sweeps    bit 0: each smoothing sweep of fmg_lin does both colours
//                   in one launch, the second colour with the block's ghost
//                   cells and reflux fluxes as they were before the sweep
//                   (k_relax_bulk FUSED, k_relax_tiled with ipass 0); bit 1:
//                   the same for the sweeps of vmg_fas; clear: the
//                   reference's two colour launches with a ghost refresh
//                   between them (fmg_poisson.F90:160-165, vmg_poisson.F90:114-115)
//   local_sweeps    full sweeps of each fused launch on the staged block
//                   (1 to 3; the ghost cells stay as staged between them)
//   key: element size 4, block edge NI, level -1, kind -1
// Text form, one entry per line (blank lines and lines starting with '#'
// are skipped):
//   <knob> <element bytes> <n> <level> <kind> <choice>
// e.g. "ghost_fill 4 8 2 -1 1".  Unknown knobs, malformed lines and choices
// outside a knob's candidates are rejected.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

namespace sfm {

enum TuneKnob {
    kKnobGhostFill = 0, kKnobRelaxThreads = 1, kKnobResidBpc = 2,
    kKnobFmgCycles = 3, kKnobFmgSweeps = 4, kKnobVmgSweeps = 5, kKnobBaseCorr = 6,
    kKnobBaseCtas = 7, kKnobBaseWide = 8, kKnobFusedSweep = 9, kKnobLocalSweeps = 10, kKnobCount = 11
};
inline const char *tune_knob_name(int k) {
    switch (k) {
        case kKnobGhostFill: return "ghost_fill";
        case kKnobRelaxThreads: return "relax_threads";
        case kKnobResidBpc: return "resid_bpc";
        case kKnobFmgCycles: return "fmg_ncycle";
        case kKnobFmgSweeps: return "fmg_sweeps";
        case kKnobVmgSweeps: return "vmg_sweeps";
        case kKnobBaseCorr: return "base_corrections";
        case kKnobBaseCtas: return "base_ctas";
        case kKnobBaseWide: return "base_wide";
        case kKnobFusedSweep: return "fused_sweeps";
        case kKnobLocalSweeps: return "local_sweeps";
        default: return nullptr;
    }
}
inline bool tune_choice_ok(int knob, int v) {
    switch (knob) {
        case kKnobGhostFill: return v == 0 || v == 1;
        case kKnobRelaxThreads: return v == 256 || v == 288 || v == 512 || v == 544;
        case kKnobResidBpc: return v == 1 || v == 2 || v == 4;
        case kKnobFmgCycles: return v >= 1 && v <= 3;
        case kKnobFmgSweeps: return v >= 1 && v <= 3;
        case kKnobVmgSweeps: return v >= 1 && v <= 3;
        case kKnobBaseCorr: return v >= 1 && v <= 10;
        case kKnobBaseCtas: return v == 1 || v == 2 || v == 4 || v == 8 || v == 16;
        case kKnobBaseWide: return v == 16 || v == 32 || v == 64;
        case kKnobFusedSweep: return v >= 0 && v <= 3;
        case kKnobLocalSweeps: return v >= 1 && v <= 3;
        default: return false;
    }
}

struct TuneTable {
    // (knob, element bytes, n, level, kind) -> choice
    using Key = std::tuple<int, int, int, int, int>;
    std::map<Key, int> v;

    int get(int knob, int elem, int n, int level, int kind, int dflt) const {
        auto it = v.find(Key{knob, elem, n, level, kind});
        return it == v.end() ? dflt : it->second;
    }
    void set(int knob, int elem, int n, int level, int kind, int choice) { v[Key{knob, elem, n, level, kind}] = choice; }

    std::string text() const {
        std::string s = "# knob elem_bytes n level kind choice\n";
        char line[128];
        for (const auto &e : v) {
            std::snprintf(line, sizeof line, "%s %d %d %d %d %d\n", tune_knob_name(std::get<0>(e.first)),
                          std::get<1>(e.first), std::get<2>(e.first), std::get<3>(e.first), std::get<4>(e.first),
                          e.second);
            s += line;
        }
        return s;
    }
    // replaces the table with the entries of `t`; false (table unchanged) on
    // any malformed or out-of-range line
    bool parse(const char *t) {
        std::map<Key, int> nv;
        std::istringstream in(t ? t : "");
        std::string line;
        while (std::getline(in, line)) {
            size_t a = line.find_first_not_of(" \t\r");
            if (a == std::string::npos || line[a] == '#') continue;
            std::istringstream ls(line);
            std::string name;
            long elem, n, level, kind, choice;
            if (!(ls >> name >> elem >> n >> level >> kind >> choice)) return false;
            std::string rest;
            if (ls >> rest) return false;
            int knob = -1;
            for (int k = 0; k < kKnobCount; k++)
                if (name == tune_knob_name(k)) knob = k;
            if (knob < 0) return false;
            if ((elem != 4 && elem != 8) || n < 2 || n > 64 || (n & (n - 1)) || level < -1 || level > 30 || kind < -1 ||
                kind > 1 || !tune_choice_ok(knob, (int)choice))
                return false;
            nv[Key{knob, (int)elem, (int)n, (int)level, (int)kind}] = (int)choice;
        }
        v.swap(nv);
        return true;
    }
};

}  // namespace sfm
