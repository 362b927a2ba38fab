// Host-side set-up of a PIAFS simulation from its input deck.
//
// Mirrors the reference's initialisation sequence for the hot path
// (src/Simulation/ReadInputs.c, Initialize.c, InitialSolution.c,
// InitializeBoundaries.c, InitializeSolvers.c, InitializePhysics.c and the
// model/chemistry initialisers) and produces the flat parameters, grid,
// initial state and boundary zones the device path consumes.
#pragma once
#include <map>
#include <string>
#include <vector>
#include "common.cuh"
#include "kernels.h"

namespace piafs {

// A sponge zone (BCSponge.c): inside the box [is, ie) of interior points the
// source gets -sigma_i (u - uref), sigma ramping linearly along `dim`.
struct SpongeZone {
  int dim, face;
  int is[2], ie[2];
  std::vector<double> sigma;   // per index along dim, is[dim] .. ie[dim]-1
  std::vector<double> uref;    // nvars
};

struct Deck {
  // solver.inp (ReadInputs.c:202-229 defaults)
  int ndims = 1, nvars = 1, ghosts = 1;
  std::vector<int> size;
  int n_iter = 0, restart_iter = 0, screen_op_iter = 1, file_op_iter = 1000;
  double dt = 0.0;
  std::string time_scheme = "euler", time_scheme_type = " ", hyp_space_scheme = "1", hyp_interp_type = "characteristic";
  std::string par_space_scheme = "2", ip_file_type = "ascii", op_file_format = "text", op_overwrite = "no";
  std::string model = "none", input_mode = "serial", output_mode = "serial", conservation_check = "no";
  // physics.inp
  double gamma = 1.4, Pr = 0.72, Re = -1.0, Tref = 273.15, T0 = 275.0, TS = 110.4, TA = 245.4, TB = 27.6;
  std::string upwinding = "roe", include_chem = "no", write_output = "yes";
  // weno.inp
  int mapped = 0, borges = 0, yc = 0, no_limiting = 0;
  double weno_eps = 1e-6;
  // derived
  double bc_gamma = 1.4;      // wall BCs keep the physics.inp gamma
  int nstages = 1;
  double A[MAX_STAGES * MAX_STAGES] = {0}, b[MAX_STAGES] = {0}, c[MAX_STAGES] = {0};
  // chemistry (normalised), valid if chem
  bool chem = false;
  int nz = 1;
  std::string write_all_zlocs = "yes";   // chemistry.inp: species files for every layer, or the last
  bool write_species = false;            // the model writes op_species_z*.bin beside the solution
  double chem_gamma = 0, kn[11] = {0}, qn[11] = {0}, I0 = 0, ch_c = 0, ch_h = 0, ch_nu = 0, n_O2 = 0;
  double t_start_norm = 0, t_pulse_norm = 0, sO3 = 0, dz = 0;
  double L_ref = 0, kg = 0, IA = 1, IB = 1, IC = 0;
  // grid and fields (host, reference layout)
  std::vector<double> x;        // ghosted coordinates, dims concatenated
  std::vector<double> dxinv;    // ghosted 1/dx, dims concatenated
  std::vector<double> grid;     // interior coordinates, dims concatenated (for output)
  std::vector<double> u0;       // AoS with ghosts
  std::vector<double> imap;     // ghosted (chemistry only)
  std::vector<Zone> zones;
  std::vector<std::vector<double>> zone_vals;   // per zone: the values Zone::val points to on the device
  std::vector<SpongeZone> sponges;
  // row slab of a decomposed grid: its first row in the whole grid and the
  // whole grid's rows (0, 0: not a slab)
  int slab_j0 = 0, slab_N1 = 0;
};

// The zones' values (Zone::val) packed in one array; off[z] is zone z's offset.
inline std::vector<double> pack_zone_values(const Deck& d, std::vector<size_t>& off) {
  std::vector<double> v;
  off.assign(d.zone_vals.size(), 0);
  for (size_t z = 0; z < d.zone_vals.size(); z++) {
    off[z] = v.size();
    v.insert(v.end(), d.zone_vals[z].begin(), d.zone_vals[z].end());
  }
  return v;
}
// Point each zone that has values at its place in `dev` (device copy of
// pack_zone_values).
inline void bind_zone_values(const Deck& d, const std::vector<size_t>& off, const double* dev, Zone* zones) {
  for (size_t z = 0; z < d.zone_vals.size(); z++) zones[z].val = d.zone_vals[z].empty() ? nullptr : dev + off[z];
}

// Parse the deck in `dir`.  Returns 0 on success, otherwise a PIAFS_ERR_*
// code with a message in `err`.
int read_deck(const std::string& dir, Deck& d, std::string& err);
// A deck held in memory: the key files (solver.inp, boundary.inp,
// physics.inp, chemistry.inp, weno.inp) by name and the interior grid
// (coordinates of each dimension, concatenated).  read_deck_memory parses it
// like read_deck and leaves u0 and imap empty for the caller to generate.
struct DeckMemory {
  std::map<std::string, std::string> files;
  std::vector<double> grid;
};
int read_deck_memory(const DeckMemory& m, Deck& d, std::string& err);
// Flat device parameters from a parsed deck.
int make_params(const Deck& d, DevParams& P, std::string& err);
// The exact solution exact.inp of a deck directory (ExactSolution.c: same
// format as initial.inp), interior points in output order; found = false
// when the file is absent.
int read_exact(const std::string& dir, const Deck& d, std::vector<double>& u_interior, bool& found,
               std::string& err);
// The options of a filled deck that lie outside the GPU path, as read_deck
// refuses them; 0 or a PIAFS_ERR_* code with a message in `err`.
int check_deck(const Deck& d, std::string& err);
// Rows [rank n1, (rank + 1) n1) of a 2D deck's grid, n1 = N1 / nranks (a row
// slab of a grid decomposed along y), as a deck of its own: coordinates,
// 1/dx, initial state and intensity map of the slab's rows with their ghost
// rows, the boundary zones that touch the slab (y-face zones on the first
// and last slab only; periodic y-face zones dropped, as the neighbouring
// slabs' rows fill those ghosts).  Sets periodic_y when the grid is periodic
// along y.
int restrict_rows(const Deck& d, int rank, int nranks, Deck& out, bool& periodic_y, std::string& err);
// Write an op_*.bin file (WriteBinary.c:37-93) from the interior AoS field of
// nvars variables (the deck's by default).
int write_binary(const std::string& path, const Deck& d, const double* u_interior, std::string& err,
                 int nvars = -1);

}  // namespace piafs

// A simulation object (api.cu) from a filled deck: device arrays, initial
// state u0 at time restart_iter x dt.  Returns PIAFS_OK or a PIAFS_ERR_*
// code (message in piafs_gpu_last_error()).
struct piafs_gpu_sim;
namespace piafs {
int create_sim(Deck&& deck, int precision, piafs_gpu_sim** out);
}  // namespace piafs
