// Oracle harness around the reference Lunar solver (test infrastructure).
//
// Runs the reference's own set-up exactly as Z4_Lunar/main.cpp:23-212 does
// (Param, Grid_Preprocess, build_topology, Field + the same field
// registrations, Halo + the same halo registrations, LunarSolver), then,
// instead of LunarSolver::Advance(), drives the solver's own member
// functions and dumps fields in the MPCNSRST v1 layout
// (src/5_io/IOModule_Bin.cpp:168-233) so the Python side reads one format.
//
// Usage (run inside a case directory holding ./CASE):
//   ref_lunar geom  <out.bin>                      geometry + node coordinates
//   ref_lunar run   <state.rst> <nsteps> <prefix>  state after each StepOnce
//   ref_lunar rk2   <state.rst> <nsteps> <prefix>  state after each SSP-RK2 step of two Euler stages
//   ref_lunar probe <state.rst> <group> <out.bin>  index-encoded Sync(group)
//   ref_lunar hall <state.rst> <out.bin>           Hall edge EMF of the state
//   ref_lunar hallstep <state.rst> <out.bin>       one implicit Hall solve (tight tolerances)
//   ref_lunar hallrun <state.rst> <n> <prefix>     n StepOnce with the implicit Hall solve (HALL_IMPLICIT == 1)
//   ref_lunar time  <state.rst> <nsteps> [w]       wall time of the step loop (after w untimed steps)
//   ref_lunar timerk2 <state.rst> <nsteps> [w]     wall time of SSP-RK2 steps (after w untimed ones)
//   ref_lunar timehall <state.rst> <nsteps> [w]    wall time of steps with the implicit Hall solve
//
// The member functions are private in the reference; this translation unit
// alone widens access to call them (the class layout is unchanged).
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <compare>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include <csignal>
#include <execinfo.h>
#include <unistd.h>

#include <mpi.h>
#include <petscksp.h>
#include <petscsnes.h>

#define private public
#define protected public
#include "1_grid/1_MPCNS_Grid.h"
#include "0_basic/MPI_WRAPPER.h"
#include "2_topology/2_MPCNS_Topology.h"
#include "3_field/2_MPCNS_Field.h"
#include "4_halo/1_MPCNS_Halo.h"
#include "LunarSolver.h"
#include "2_topology/2_MPCNS_Topology_Equiv.h"
#include "4_halo/1_MPCNS_Halo_EdgeOwner.h"
#undef private
#undef protected

namespace
{

void wr_i32(std::ofstream &o, int32_t v) { o.write(reinterpret_cast<const char *>(&v), 4); }
void wr_f64(std::ofstream &o, double v) { o.write(reinterpret_cast<const char *>(&v), 8); }
void wr_str(std::ofstream &o, const std::string &s)
{
    wr_i32(o, int32_t(s.size()));
    o.write(s.data(), std::streamsize(s.size()));
}

// location code as the restart writer stores it (src/5_io/IOModule_Bin.cpp:62-85)
int loc_code(StaggerLocation l)
{
    switch (l)
    {
    case StaggerLocation::Cell:
        return 0;
    case StaggerLocation::FaceXi:
        return 1;
    case StaggerLocation::FaceEt:
        return 2;
    case StaggerLocation::FaceZe:
        return 3;
    case StaggerLocation::EdgeXi:
        return 4;
    case StaggerLocation::EdgeEt:
        return 5;
    case StaggerLocation::EdgeZe:
        return 6;
    default:
        return 7;
    }
}

// One dump entry: either a registered field or a node-coordinate array.
struct DumpItem
{
    std::string name;
    int loc;
    int ncomp;
    int nghost;
    std::function<void(int ib, Int3 &lo, Int3 &hi, bool &active)> extent;
    std::function<double(int ib, int i, int j, int k, int m)> value;
};

void write_dump(const std::string &path, int step, double time, int nblock, const std::vector<DumpItem> &items)
{
    std::ofstream out(path, std::ios::binary);
    if (!out)
    {
        std::fprintf(stderr, "cannot open %s\n", path.c_str());
        std::exit(2);
    }
    const char magic[8] = {'M', 'P', 'C', 'N', 'S', 'R', 'S', 'T'};
    out.write(magic, 8);
    wr_i32(out, 1);
    wr_i32(out, step);
    wr_f64(out, time);
    wr_i32(out, nblock);
    wr_i32(out, int32_t(items.size()));
    for (const auto &it : items)
    {
        wr_str(out, it.name);
        wr_i32(out, it.loc);
        wr_i32(out, it.ncomp);
        wr_i32(out, it.nghost);
        for (int ib = 0; ib < nblock; ++ib)
        {
            Int3 lo{}, hi{};
            bool active = false;
            it.extent(ib, lo, hi, active);
            wr_i32(out, lo.i);
            wr_i32(out, lo.j);
            wr_i32(out, lo.k);
            wr_i32(out, hi.i);
            wr_i32(out, hi.j);
            wr_i32(out, hi.k);
            wr_i32(out, active ? 1 : 0);
            if (!active)
                continue;
            for (int i = lo.i; i < hi.i; ++i)
                for (int j = lo.j; j < hi.j; ++j)
                    for (int k = lo.k; k < hi.k; ++k)
                        for (int m = 0; m < it.ncomp; ++m)
                            wr_f64(out, it.value(ib, i, j, k, m));
        }
    }
}

DumpItem field_item(Field *fld, const std::string &name)
{
    const int fid = fld->field_id(name);
    const FieldDescriptor &d = fld->descriptor(fid);
    DumpItem it;
    it.name = name;
    it.loc = loc_code(d.location);
    it.ncomp = d.ncomp;
    it.nghost = d.nghost;
    it.extent = [fld, fid](int ib, Int3 &lo, Int3 &hi, bool &active)
    {
        FieldBlock &fb = fld->field(fid, ib);
        lo = fb.get_lo();
        hi = fb.get_hi();
        active = fb.is_allocated();
    };
    it.value = [fld, fid](int ib, int i, int j, int k, int m) { return fld->field(fid, ib)(i, j, k, m); };
    return it;
}

// Node coordinates with the reference's ghost nodes (ngg+1 layers), as a
// pseudo-field with location code 1 (Node) and 3 components (x, y, z).
DumpItem node_item(Grid *grd)
{
    DumpItem it;
    it.name = "X_node";
    it.loc = loc_code(StaggerLocation::Node);
    it.ncomp = 3;
    it.nghost = grd->ngg + 1;
    it.extent = [grd](int ib, Int3 &lo, Int3 &hi, bool &active)
    {
        const Block &b = grd->grids(ib);
        const int g = grd->ngg + 1;
        lo = Int3{-g, -g, -g};
        hi = Int3{b.mx + 1 + g, b.my + 1 + g, b.mz + 1 + g};
        active = true;
    };
    it.value = [grd](int ib, int i, int j, int k, int m)
    {
        Block &b = grd->grids(ib);
        if (m == 0)
            return b.x(i, j, k);
        if (m == 1)
            return b.y(i, j, k);
        return b.z(i, j, k);
    };
    return it;
}

struct Harness
{
    Param *par = nullptr;
    Grid *grd = nullptr;
    TOPO::Topology topology;
    TOPO::TopologyEquiv topo_equiv;
    Field *fld = nullptr;
    Halo *hal = nullptr;
    HALO_OWNER::EdgeOwnerSyncPattern edge_owner_pattern;
    std::unique_ptr<LunarSolver> solver;
    bool topo_only = false;

    // Z4_Lunar/main.cpp:43-212, unchanged in substance.
    void setup()
    {
        int myid = 0;
        par = new Param;
        par->ReadParam(myid);
        grd = new Grid;
        grd->Grid_Preprocess(par);
        topology = TOPO::build_topology(*grd, myid, par->GetInt("dimension"));
        if (topo_only)
            return;
        TOPO::build_topology_equiv(topology, *grd, myid, par->GetInt("dimension"), topo_equiv);
        const int ngg = par->GetInt("ngg");
        fld = new Field(grd, par, ngg);
        fld->register_field({"U_H", StaggerLocation::Cell, 5, ngg, "Fluid"});
        fld->register_field({"B_xi", StaggerLocation::FaceXi, 1, ngg});
        fld->register_field({"B_eta", StaggerLocation::FaceEt, 1, ngg});
        fld->register_field({"B_zeta", StaggerLocation::FaceZe, 1, ngg});
        fld->register_field({"E_xi", StaggerLocation::EdgeXi, 1, ngg});
        fld->register_field({"E_eta", StaggerLocation::EdgeEt, 1, ngg});
        fld->register_field({"E_zeta", StaggerLocation::EdgeZe, 1, ngg});
        fld->register_field({"Ehall_xi", StaggerLocation::EdgeXi, 1, ngg});
        fld->register_field({"Ehall_eta", StaggerLocation::EdgeEt, 1, ngg});
        fld->register_field({"Ehall_zeta", StaggerLocation::EdgeZe, 1, ngg});
        fld->register_field({"Eres_xi", StaggerLocation::EdgeXi, 1, ngg});
        fld->register_field({"Eres_eta", StaggerLocation::EdgeEt, 1, ngg});
        fld->register_field({"Eres_zeta", StaggerLocation::EdgeZe, 1, ngg});
        fld->register_field({"Eface_xi", StaggerLocation::FaceXi, 3, ngg});
        fld->register_field({"Eface_eta", StaggerLocation::FaceEt, 3, ngg});
        fld->register_field({"Eface_zeta", StaggerLocation::FaceZe, 3, ngg});
        fld->register_field({"J_xi", StaggerLocation::EdgeXi, 1, ngg});
        fld->register_field({"J_eta", StaggerLocation::EdgeEt, 1, ngg});
        fld->register_field({"J_zeta", StaggerLocation::EdgeZe, 1, ngg});
        fld->register_field({"J_cell", StaggerLocation::Cell, 3, ngg});
        fld->register_field({"dE_xi", StaggerLocation::EdgeXi, 1, ngg});
        fld->register_field({"dE_eta", StaggerLocation::EdgeEt, 1, ngg});
        fld->register_field({"dE_zeta", StaggerLocation::EdgeZe, 1, ngg});
        fld->register_field({"dB_xi", StaggerLocation::FaceXi, 1, ngg});
        fld->register_field({"dB_eta", StaggerLocation::FaceEt, 1, ngg});
        fld->register_field({"dB_zeta", StaggerLocation::FaceZe, 1, ngg});
        fld->register_field({"dJ_xi", StaggerLocation::EdgeXi, 1, ngg});
        fld->register_field({"dJ_eta", StaggerLocation::EdgeEt, 1, ngg});
        fld->register_field({"dJ_zeta", StaggerLocation::EdgeZe, 1, ngg});
        fld->register_field({"dJ_cell", StaggerLocation::Cell, 3, ngg});
        fld->register_field({"dEpre_xi", StaggerLocation::EdgeXi, 1, ngg});
        fld->register_field({"dEpre_eta", StaggerLocation::EdgeEt, 1, ngg});
        fld->register_field({"dEpre_zeta", StaggerLocation::EdgeZe, 1, ngg});
        fld->register_field({"Badd_xi", StaggerLocation::FaceXi, 1, ngg});
        fld->register_field({"Badd_eta", StaggerLocation::FaceEt, 1, ngg});
        fld->register_field({"Badd_zeta", StaggerLocation::FaceZe, 1, ngg});
        fld->register_field({"B_cell", StaggerLocation::Cell, 3, ngg});
        fld->register_field({"Bind_cell", StaggerLocation::Cell, 3, ngg});
        fld->register_field({"U_plus", StaggerLocation::Cell, 3, ngg});
        fld->register_field(FieldDescriptor{"PV_H", StaggerLocation::Cell, 5, ngg, "Fluid"});
        fld->register_field({"F_xi", StaggerLocation::FaceXi, 5, 0, "Fluid"});
        fld->register_field({"F_eta", StaggerLocation::FaceEt, 5, 0, "Fluid"});
        fld->register_field({"F_zeta", StaggerLocation::FaceZe, 5, 0, "Fluid"});
        fld->register_field(FieldDescriptor{"divB", StaggerLocation::Cell, 1, 1});
        fld->register_field(FieldDescriptor{"RHS_H", StaggerLocation::Cell, 5, 0, "Fluid"});
        fld->register_field(FieldDescriptor{"RHS_B_xi", StaggerLocation::FaceXi, 1, 0});
        fld->register_field(FieldDescriptor{"RHS_B_eta", StaggerLocation::FaceEt, 1, 0});
        fld->register_field(FieldDescriptor{"RHS_B_zeta", StaggerLocation::FaceZe, 1, 0});
        fld->register_field(FieldDescriptor{"RHS_Bres_xi", StaggerLocation::FaceXi, 1, 0});
        fld->register_field(FieldDescriptor{"RHS_Bres_eta", StaggerLocation::FaceEt, 1, 0});
        fld->register_field(FieldDescriptor{"RHS_Bres_zeta", StaggerLocation::FaceZe, 1, 0});

        hal = new Halo(fld, &topology);
        for (const char *fn : {"U_H", "U_plus", "B_xi", "B_eta", "B_zeta", "Badd_xi", "Badd_eta", "Badd_zeta",
                               "E_xi", "E_eta", "E_zeta", "J_xi", "J_eta", "J_zeta", "Ehall_xi", "Ehall_eta",
                               "Ehall_zeta", "Eres_xi", "Eres_eta", "Eres_zeta", "dB_xi", "dB_eta", "dB_zeta",
                               "dE_xi", "dE_eta", "dE_zeta", "dJ_xi", "dJ_eta", "dJ_zeta", "dJ_cell"})
        {
            std::string s(fn);
            hal->register_halo_field(s, HaloLevel::Vertex);
        }
        hal->build_registered_patterns();
        HALO_OWNER::build_edge_owner_sync_pattern(topo_equiv, edge_owner_pattern);

        solver = std::make_unique<LunarSolver>(grd, &topology, fld, hal, par, &topo_equiv, &edge_owner_pattern);
    }

    // Load U_H and B_xi/B_eta/B_zeta from an MPCNSRST file, then fill their
    // ghosts with the reference's own Sync so every derived field starts
    // from a consistent state.
    void load_state(const std::string &path)
    {
        solver->io_.Change_RestartPath(path);
        solver->io_.ReadRestartBinFile();
        solver->lunar_bound_.Sync("Ucell");
        solver->lunar_bound_.Sync("Bface");
    }
};

const std::vector<std::string> &geom_fields()
{
    static const std::vector<std::string> v = {
        "Jac", "JDxi", "JDet", "JDze", "beta_xi", "beta_eta", "beta_zeta", "alpha_xi", "alpha_eta",
        "alpha_zeta", "dr_xi", "dr_eta", "dr_zeta", "Area_xi", "Area_eta", "Area_zeta", "dl_xi", "dl_eta",
        "dl_zeta", "Bcell_from_Bface_w", "Jcell_from_Jedge_w", "Badd_xi", "Badd_eta", "Badd_zeta"};
    return v;
}

const std::vector<std::string> &state_fields()
{
    static const std::vector<std::string> v = {
        "U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "U_plus", "B_cell", "Bind_cell", "J_xi", "J_eta", "J_zeta",
        "J_cell", "E_xi", "E_eta", "E_zeta", "Eface_xi", "Eface_eta", "Eface_zeta", "RHS_H", "RHS_B_xi",
        "RHS_B_eta", "RHS_B_zeta", "divB", "Eres_xi", "Eres_eta", "Eres_zeta"};
    return v;
}

int cmd_geom(Harness &h, const std::string &out)
{
    std::vector<DumpItem> items;
    for (const auto &n : geom_fields())
        items.push_back(field_item(h.fld, n));
    items.push_back(node_item(h.grd));
    write_dump(out, 0, 0.0, h.fld->num_blocks(), items);
    return 0;
}

void dump_state(Harness &h, const std::string &path, const std::vector<std::string> &extra = {})
{
    std::vector<DumpItem> items;
    for (const auto &n : state_fields())
        items.push_back(field_item(h.fld, n));
    for (const auto &n : extra)
        items.push_back(field_item(h.fld, n));
    // dt of the step just taken, as a 1x1x1 pseudo-field
    DumpItem dti;
    dti.name = "dt";
    dti.loc = -1;
    dti.ncomp = 1;
    dti.nghost = 0;
    LunarSolver *s = h.solver.get();
    dti.extent = [](int, Int3 &lo, Int3 &hi, bool &active)
    {
        lo = Int3{0, 0, 0};
        hi = Int3{1, 1, 1};
        active = true;
    };
    dti.value = [s](int, int, int, int, int) { return s->dt; };
    items.push_back(dti);
    write_dump(path, s->run_data_->step, s->run_data_->time, h.fld->num_blocks(), items);
}

// The reference's output-step diagnostics after nsteps StepOnce: calc_divB,
// then PrintMinMaxDiagnostics_ (its own printf lines on stdout)
int cmd_diag(Harness &h, const std::string &state, int nsteps)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    for (int n = 0; n < nsteps; ++n)
        s.StepOnce();
    s.calc_divB();
    s.PrintMinMaxDiagnostics_();
    return 0;
}

int cmd_run(Harness &h, const std::string &state, int nsteps, const std::string &prefix)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    // divB as the reference computes it at output steps (UpdateControlAndOutput)
    s.calc_divB();
    dump_state(h, prefix + "_0000.bin");
    for (int n = 1; n <= nsteps; ++n)
    {
        s.StepOnce();
        s.calc_divB();
        char buf[32];
        std::snprintf(buf, sizeof(buf), "_%04d.bin", n);
        dump_state(h, prefix + buf);
    }
    return 0;
}

// One forward-Euler stage of StepOnce at the solver's current dt
// (Z4_Lunar/src/LunarSolver_Driver.cpp:21-48 without Compute_Timestep): the
// reference's own RHS, CT induction, update and resistive part.
void euler_stage(LunarSolver &s)
{
    s.ZeroRHS_();
    s.Scheme_U_();
    s.AddSourceToRHS_Fluid();
    s.AssembleRHS_Induction_CT_();
    s.ApplyUpdate_Euler_();
    if (s.resist_control.use_implicit_lunar_resistance)
    {
        s.lunar_bound_.Sync("Bface");
        s.SolveImplicitResistiveDiffusion_(s.dt);
    }
    else
        s.ResistiveDiffusionSubcycles_();
}

// The state fields the Euler update writes, on the inner points it writes
// (ApplyUpdate_Euler_, Z4_Lunar/src/physics/LunarSolver_Advance.cpp:61-122)
std::vector<FieldBlock *> state_blocks(Harness &h, int ib)
{
    LunarSolver &s = *h.solver;
    return {&h.fld->field(s.fid_.fid_U_H, ib), &h.fld->field(s.fid_.fid_B.xi, ib),
            &h.fld->field(s.fid_.fid_B.eta, ib), &h.fld->field(s.fid_.fid_B.zeta, ib)};
}

template <class F> void for_inner(FieldBlock &f, F fn)
{
    const Int3 lo = f.inner_lo(), hi = f.inner_hi();
    const int nc = f.descriptor().ncomp;
    for (int i = lo.i; i < hi.i; ++i)
        for (int j = lo.j; j < hi.j; ++j)
            for (int k = lo.k; k < hi.k; ++k)
                for (int m = 0; m < nc; ++m)
                    fn(f(i, j, k, m));
}

// SSP-RK2 (Shu and Osher, 1988) composed from two of the reference's Euler
// stages at the dt of the step's start: U1 = U^n + dt L(U^n), then
// U^{n+1} = 0.5 (U^n + (U1 + dt L(U1))) on the inner points, with the
// reference's syncs and derived fields after each stage.  The reference has
// no multi-stage integrator; this is the composition the device's
// mhd_set_integrator(MHD_INTEGRATOR_SSPRK2) follows.
void rk2_step(Harness &h)
{
    LunarSolver &s = *h.solver;
    const int nb = h.fld->num_blocks();
    s.Compute_Timestep();
    std::vector<std::vector<double>> u0(static_cast<size_t>(nb));
    for (int ib = 0; ib < nb; ++ib)
        for (FieldBlock *f : state_blocks(h, ib))
            for_inner(*f, [&](double &x) { u0[size_t(ib)].push_back(x); });
    euler_stage(s);
    s.lunar_bound_.Sync("Ucell");
    s.lunar_bound_.Sync("Bface");
    s.UpdateDerivedFields_();
    euler_stage(s);
    for (int ib = 0; ib < nb; ++ib)
    {
        size_t q = 0;
        for (FieldBlock *f : state_blocks(h, ib))
            for_inner(*f, [&](double &x) {
                x = 0.5 * (u0[size_t(ib)][q] + x);
                ++q;
            });
    }
    s.run_data_->dt = s.dt;
    s.run_data_->time += s.dt;
    s.run_data_->step += 1;
    s.lunar_bound_.Sync("Ucell");
    s.lunar_bound_.Sync("Bface");
    s.UpdateDerivedFields_();
}

int cmd_rk2(Harness &h, const std::string &state, int nsteps, const std::string &prefix)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    s.calc_divB();
    dump_state(h, prefix + "_0000.bin");
    for (int n = 1; n <= nsteps; ++n)
    {
        rk2_step(h);
        s.calc_divB();
        char buf[32];
        std::snprintf(buf, sizeof(buf), "_%04d.bin", n);
        dump_state(h, prefix + buf);
    }
    return 0;
}

// StepOnce as the reference compiles it with HALL_IMPLICIT == 1
// (Z4_Lunar/src/LunarSolver_Driver.cpp:21-92): the Euler stage, then the
// implicit Hall solve at the step's dt (SolveOneStep) and calc_Bcell, then
// the step's closing syncs and derived fields.  The nonlinear solve is
// tightened to ||F|| <= 1e-12 ||F0|| so that its root is pinned closely.
void hall_step(LunarSolver &s)
{
    s.Compute_Timestep();
    euler_stage(s);
    s.hall_implicit_.SolveOneStep(s.dt, false);
    s.calc_Bcell();
    s.run_data_->dt = s.dt;
    s.run_data_->time += s.dt;
    s.run_data_->step += 1;
    s.lunar_bound_.Sync("Ucell");
    s.lunar_bound_.Sync("Bface");
    s.UpdateDerivedFields_();
}

int cmd_hallrun(Harness &h, const std::string &state, int nsteps, const std::string &prefix)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    SNESSetTolerances(s.hall_implicit_.snes_, 1e-30, 1e-12, 1e-30, 200, PETSC_DEFAULT);
    s.calc_divB();
    const std::vector<std::string> ehall = {"Ehall_xi", "Ehall_eta", "Ehall_zeta"};
    dump_state(h, prefix + "_0000.bin", ehall);
    for (int n = 1; n <= nsteps; ++n)
    {
        hall_step(s);
        s.calc_divB();
        char buf[32];
        std::snprintf(buf, sizeof(buf), "_%04d.bin", n);
        dump_state(h, prefix + buf, ehall);
    }
    return 0;
}

// Every field of the group is overwritten with value = block*2^32 + AoS
// offset + 1 (exact in a double), then the reference Sync(group) runs; the
// dump therefore records, for every point, which original point it was copied
// from (or a non-integer value where a handler computed it).
int cmd_probe(Harness &h, const std::string &state, const std::string &group, const std::string &out)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    auto git = s.lunar_bound_.groups_.find(group);
    if (git == s.lunar_bound_.groups_.end())
    {
        std::fprintf(stderr, "unknown group %s\n", group.c_str());
        return 2;
    }
    std::vector<DumpItem> items;
    for (const auto &fn : git->second.fields)
    {
        const int fid = h.fld->field_id(fn);
        const int ncomp = h.fld->descriptor(fid).ncomp;
        for (int ib = 0; ib < h.fld->num_blocks(); ++ib)
        {
            FieldBlock &fb = h.fld->field(fid, ib);
            if (!fb.is_allocated())
                continue;
            const Int3 lo = fb.get_lo(), hi = fb.get_hi();
            const int64_t nj = hi.j - lo.j, nk = hi.k - lo.k;
            for (int i = lo.i; i < hi.i; ++i)
                for (int j = lo.j; j < hi.j; ++j)
                    for (int k = lo.k; k < hi.k; ++k)
                        for (int m = 0; m < ncomp; ++m)
                        {
                            const int64_t off = (((int64_t(i - lo.i) * nj + (j - lo.j)) * nk + (k - lo.k)) * ncomp + m);
                            fb(i, j, k, m) = double(int64_t(ib) * (int64_t(1) << 32) + off + 1);
                        }
        }
        items.push_back(field_item(h.fld, fn));
    }
    s.lunar_bound_.Sync(group);
    write_dump(out, 0, 0.0, h.fld->num_blocks(), items);
    return 0;
}

// Topology summary: physical, inner, edge and vertex patches (text).
int cmd_topo(Harness &h, const std::string &out)
{
    std::ofstream o(out);
    const auto &t = h.topology;
    for (const auto &p : t.physical_patches)
        o << "physical " << p.this_block << " " << p.bc_name << " dir " << p.direction << " box " << p.this_box_node.lo.i
          << " " << p.this_box_node.lo.j << " " << p.this_box_node.lo.k << " " << p.this_box_node.hi.i << " "
          << p.this_box_node.hi.j << " " << p.this_box_node.hi.k << "\n";
    for (const auto &p : t.inner_patches)
        o << "inner " << p.this_block << "->" << p.nb_block << " [" << p.this_block_name << "|" << p.nb_block_name
          << "] coupling " << p.is_coupling << " perm " << p.trans.perm[0] << p.trans.perm[1] << p.trans.perm[2]
          << " sign " << p.trans.sign[0] << " " << p.trans.sign[1] << " " << p.trans.sign[2] << " off "
          << p.trans.offset.i << " " << p.trans.offset.j << " " << p.trans.offset.k << "\n";
    o << "inner_edge " << t.inner_edge_patches.size() << " physical_edge " << t.physical_edge_patches.size()
      << " inner_vertex " << t.inner_vertex_patches.size() << " physical_vertex " << t.physical_vertex_patches.size()
      << "\n";
    return 0;
}

// Edge equivalence: alias -> owner copies (with sign) and, when the solver
// built its implicit resistive system, its DOF list in solve order with eta.
int cmd_owners(Harness &h, const std::string &out)
{
    std::ofstream o(out);
    o << std::setprecision(17);
    for (const auto &it : h.edge_owner_pattern.local_alias)
        o << "alias " << it.rep.gblock << " " << it.rep.dir << " " << it.rep.i << " " << it.rep.j << " " << it.rep.k
          << " owner " << it.owner.gblock << " " << it.owner.dir << " " << it.owner.i << " " << it.owner.j << " "
          << it.owner.k << " sign " << int(it.sign) << "\n";
    LunarSolver &s = *h.solver;
    for (const auto &d : s.implicit_resistive_dofs_)
        o << "dof " << d.edge.gblock << " " << d.edge.dir << " " << d.edge.i << " " << d.edge.j << " " << d.edge.k
          << " eta " << d.eta << "\n";
    o << "n_owner " << h.topo_equiv.n_local_edge_owner << "\n";
    return 0;
}

// The Hall edge EMF of a state (LunarSolver::BuildHallFaceEMF_Rusanov_diff_,
// after the derived fields), with the fields it reads.
int cmd_hall(Harness &h, const std::string &state, const std::string &out)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    s.BuildHallFaceEMF_Rusanov_diff_();
    std::vector<DumpItem> items;
    for (const char *n : {"Ehall_xi", "Ehall_eta", "Ehall_zeta", "B_cell", "J_cell", "U_H", "B_xi", "B_eta", "B_zeta"})
        items.push_back(field_item(h.fld, n));
    write_dump(out, 0, 0.0, h.fld->num_blocks(), items);
    return 0;
}

// One implicit Hall solve (ImplicitHallSolver::SolveOneStep with the CFL dt
// of the state, then calc_Bcell as StepOnce does), the nonlinear solve
// tightened to ||F|| <= 1e-12 ||F0|| so that its root is pinned closely.
int cmd_hallstep(Harness &h, const std::string &state, const std::string &out)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    s.Compute_Timestep();
    SNESSetTolerances(s.hall_implicit_.snes_, 1e-30, 1e-12, 1e-30, 200, PETSC_DEFAULT);
    s.hall_implicit_.SolveOneStep(s.dt, true);
    s.calc_Bcell();
    std::vector<DumpItem> items;
    for (const char *n : {"B_xi", "B_eta", "B_zeta", "Ehall_xi", "Ehall_eta", "Ehall_zeta", "B_cell", "RHS_B_xi",
                          "RHS_B_eta", "RHS_B_zeta"})
        items.push_back(field_item(h.fld, n));
    DumpItem dti;
    dti.name = "dt";
    dti.loc = -1;
    dti.ncomp = 1;
    dti.nghost = 0;
    dti.extent = [](int, Int3 &lo, Int3 &hi, bool &active)
    {
        lo = Int3{0, 0, 0};
        hi = Int3{1, 1, 1};
        active = true;
    };
    dti.value = [&s](int, int, int, int, int) { return s.dt; };
    items.push_back(dti);
    write_dump(out, 0, 0.0, h.fld->num_blocks(), items);
    return 0;
}

// wall time of `nsteps` StepOnce after `warmup` untimed ones, for timing
int cmd_time(Harness &h, const std::string &state, int nsteps, int warmup)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    for (int n = 0; n < warmup; ++n) // untimed
        s.StepOnce();
    int64_t cells = 0;
    for (int ib = 0; ib < h.fld->num_blocks(); ++ib)
    {
        FieldBlock &U = h.fld->field(s.fid_.fid_U_H, ib);
        const Int3 lo = U.inner_lo(), hi = U.inner_hi();
        cells += int64_t(hi.i - lo.i) * (hi.j - lo.j) * (hi.k - lo.k);
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (int n = 0; n < nsteps; ++n)
        s.StepOnce();
    const auto t1 = std::chrono::steady_clock::now();
    const double sec = std::chrono::duration<double>(t1 - t0).count();
    std::printf("{\"cells\": %lld, \"steps\": %d, \"seconds\": %.9f, \"cell_updates_per_s\": %.6e}\n",
                (long long)cells, nsteps, sec, double(cells) * nsteps / sec);
    return 0;
}

// wall time of `nsteps` SSP-RK2 steps (rk2_step), for timing
int cmd_timerk2(Harness &h, const std::string &state, int nsteps, int warmup)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    for (int n = 0; n < warmup; ++n) // untimed
        rk2_step(h);
    int64_t cells = 0;
    for (int ib = 0; ib < h.fld->num_blocks(); ++ib)
    {
        FieldBlock &U = h.fld->field(s.fid_.fid_U_H, ib);
        const Int3 lo = U.inner_lo(), hi = U.inner_hi();
        cells += int64_t(hi.i - lo.i) * (hi.j - lo.j) * (hi.k - lo.k);
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (int n = 0; n < nsteps; ++n)
        rk2_step(h);
    const auto t1 = std::chrono::steady_clock::now();
    const double sec = std::chrono::duration<double>(t1 - t0).count();
    std::printf("{\"cells\": %lld, \"steps\": %d, \"seconds\": %.9f, \"cell_updates_per_s\": %.6e}\n",
                (long long)cells, nsteps, sec, double(cells) * nsteps / sec);
    return 0;
}

// `nsteps` StepOnce as compiled with HALL_IMPLICIT == 1 (hall_step: the
// implicit Hall solve at the step's dt, Newton rtol 1e-10, then calc_Bcell,
// before the closing syncs and derived fields), for timing
int cmd_timehall(Harness &h, const std::string &state, int nsteps, int warmup)
{
    h.load_state(state);
    LunarSolver &s = *h.solver;
    s.UpdateDerivedFields_();
    SNESSetTolerances(s.hall_implicit_.snes_, 1e-50, 1e-10, 1e-30, 50, PETSC_DEFAULT);
    for (int n = 0; n < warmup; ++n) // untimed
        hall_step(s);
    int64_t cells = 0;
    for (int ib = 0; ib < h.fld->num_blocks(); ++ib)
    {
        FieldBlock &U = h.fld->field(s.fid_.fid_U_H, ib);
        const Int3 lo = U.inner_lo(), hi = U.inner_hi();
        cells += int64_t(hi.i - lo.i) * (hi.j - lo.j) * (hi.k - lo.k);
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (int n = 0; n < nsteps; ++n)
        hall_step(s);
    const auto t1 = std::chrono::steady_clock::now();
    const double sec = std::chrono::duration<double>(t1 - t0).count();
    std::printf("{\"cells\": %lld, \"steps\": %d, \"seconds\": %.9f, \"cell_updates_per_s\": %.6e}\n",
                (long long)cells, nsteps, sec, double(cells) * nsteps / sec);
    return 0;
}

} // namespace

// On abort (e.g. a failed bounds assertion in a checked build) print the
// call stack, to locate the failing reference routine.
void on_abort(int)
{
    void *frames[64];
    const int n = backtrace(frames, 64);
    backtrace_symbols_fd(frames, n, 2);
    _exit(134);
}

int main(int argc, char **argv)
{
    std::signal(SIGABRT, on_abort);
    if (argc < 3)
    {
        std::fprintf(stderr, "usage: ref_lunar geom|run|probe|time ...\n");
        return 2;
    }
    PARALLEL::mpi_initial(argc, argv);
    PetscInitialize(&argc, &argv, nullptr, nullptr);
    int rc = 0;
    {
        // the reference prints progress on stdout; keep stdout for results
        std::streambuf *saved = std::cout.rdbuf();
        std::ofstream sink("ref_harness.log");
        std::cout.rdbuf(sink.rdbuf());
        Harness h;
        if (std::string(argv[1]) == "topo")
            h.topo_only = true;
        h.setup();
        const std::string cmd = argv[1];
        if (cmd == "topo")
            rc = cmd_topo(h, argv[2]);
        else if (cmd == "owners")
            rc = cmd_owners(h, argv[2]);
        else if (cmd == "hall" && argc >= 4)
            rc = cmd_hall(h, argv[2], argv[3]);
        else if (cmd == "hallstep" && argc >= 4)
            rc = cmd_hallstep(h, argv[2], argv[3]);
        else if (cmd == "geom")
            rc = cmd_geom(h, argv[2]);
        else if (cmd == "run" && argc >= 5)
            rc = cmd_run(h, argv[2], std::atoi(argv[3]), argv[4]);
        else if (cmd == "rk2" && argc >= 5)
            rc = cmd_rk2(h, argv[2], std::atoi(argv[3]), argv[4]);
        else if (cmd == "hallrun" && argc >= 5)
            rc = cmd_hallrun(h, argv[2], std::atoi(argv[3]), argv[4]);
        else if (cmd == "probe" && argc >= 5)
            rc = cmd_probe(h, argv[2], argv[3], argv[4]);
        else if (cmd == "diag" && argc >= 4)
        {
            std::cout.rdbuf(saved);
            rc = cmd_diag(h, argv[2], std::atoi(argv[3]));
        }
        else if (cmd == "timehall" && argc >= 4)
        {
            std::cout.rdbuf(sink.rdbuf());
            rc = cmd_timehall(h, argv[2], std::atoi(argv[3]), argc >= 5 ? std::atoi(argv[4]) : 0);
        }
        else if (cmd == "timerk2" && argc >= 4)
        {
            std::cout.rdbuf(saved);
            std::cout.rdbuf(sink.rdbuf());
            rc = cmd_timerk2(h, argv[2], std::atoi(argv[3]), argc >= 5 ? std::atoi(argv[4]) : 0);
        }
        else if (cmd == "time" && argc >= 4)
        {
            std::cout.rdbuf(saved);
            std::streambuf *s2 = std::cout.rdbuf();
            // timing result goes to stdout via printf; solver chatter to the log
            std::cout.rdbuf(sink.rdbuf());
            rc = cmd_time(h, argv[2], std::atoi(argv[3]), argc >= 5 ? std::atoi(argv[4]) : 0);
            (void)s2;
        }
        else
        {
            std::fprintf(stderr, "bad command\n");
            rc = 2;
        }
        std::cout.rdbuf(saved);
    }
    PetscFinalize();
    PARALLEL::mpi_finalize();
    return rc;
}
