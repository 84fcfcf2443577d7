// Host side of a dugksFoam case without OpenFOAM: a reader for the ASCII
// files a case directory holds (constant/polyMesh, constant/Xis,
// constant/weights, constant/DVMProperties, 0/rho, 0/U, 0/T,
// system/controlDict), the flattening of the mesh into the fv addressing
// the C ABI takes (include/dugks.h), and a writer for the macro fields a
// time directory gets (src/dugksFoam.C:83 runTime.write()).
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace dugks_host {

struct FoamError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// A parsed OpenFOAM value: a word, a number, a list "( ... )", a dimension
// set "[ ... ]" or a dictionary "{ ... }".  A dictionary entry with several
// values before its ';' is a list of those values.
struct FoamValue {
    enum Kind { Word, Number, List, Dims, Dict } kind = Word;
    std::string word;
    double num = 0.0;
    std::vector<FoamValue> items;                              // List, Dims
    std::vector<std::pair<std::string, FoamValue>> entries;   // Dict, in file order

    bool is_number() const { return kind == Number; }
    const FoamValue* find(const std::string& key) const;
    const FoamValue& at(const std::string& key) const;
    // the value as a number: a number, or the last number of an entry
    // such as "R [0 2 -2 -1 0 0 0] 208.24" or "R R [..] 208.24"
    double number() const;
};

// a whole file's dictionary (the FoamFile header is kept under "FoamFile")
FoamValue read_dict(const std::string& path);

// counted lists: "N ( ... )" or "N{value}"
std::vector<double> read_scalar_list(const std::string& path);
std::vector<int64_t> read_label_list(const std::string& path);
std::vector<double> read_points(const std::string& path);                 // [n*3]
void read_faces(const std::string& path, std::vector<int64_t>& offsets, std::vector<int64_t>& labels);

struct PatchInfo {
    std::string name, type;
    int64_t start = 0, size = 0;
};
std::vector<PatchInfo> read_boundary(const std::string& path);

struct PolyMesh {
    std::vector<double> points;
    std::vector<int64_t> face_offsets, face_points, owner, neighbour;
    std::vector<PatchInfo> patches;
    int64_t n_cells = 0;
    int n_solution_dims = 3;
    int64_t n_faces() const { return static_cast<int64_t>(owner.size()); }
    int64_t n_internal() const { return static_cast<int64_t>(neighbour.size()); }
};
// n_solution_dims = 3 minus the number of non-empty patches of type empty
// constant/<mesh> of a case (polyMesh; vMesh: the velocity mesh)
PolyMesh read_polymesh(const std::string& case_dir, const std::string& mesh = "polyMesh");

// a volScalarField or volVectorField: internal values and, per patch, the
// type and the first face value (the patch values the boundary conditions use)
struct VolField {
    int ncomp = 1;
    std::vector<double> internal;   // [n_cells * ncomp]
    struct Patch {
        std::string type;
        std::vector<double> value;   // [size * ncomp], empty if the entry has none
        double pressure = 0;         // pressureIn / pressureOut entry of the patch, if any
    };
    std::map<std::string, Patch> patches;
};
VolField read_vol_field(const std::string& path, int64_t n_cells, const std::vector<PatchInfo>& patches);

// boundary condition kinds of the rho patch types (discreteVelocity::setBCtype,
// src/fvDVM/discreteVelocity/discreteVelocity.C:188-195)
// g/h surface type by the rho patch type (discreteVelocity::setBCtype,
// discreteVelocity.C:188-195): calculatedMaxwell -> MaxwellWall, farField,
// zeroGradient, fixedValue -> Mixed, symmetryPlane, symmetryMod ->
// DVMSymmetry, pressureIn, pressureOut
enum class PatchKind { Empty, MaxwellWall, FarField, ZeroGradient, Mixed, Symmetry, DVMSymmetry, PressureIn, PressureOut };
int32_t patch_type_of(PatchKind k);      // dugks_patch_type
const char* kind_name(PatchKind k);

struct Case {
    std::string dir;
    PolyMesh mesh;
    int D = 3;
    std::vector<double> xis, weights;   // one-dimensional DV set
    double xi_max = 0;
    bool macro_flux = false;            // fvDVMparas macroFlux yes
    // DV list from constant/vMesh (the VMESH build, fvDVM.C:129-277): xi = its
    // cell centres [n*3], weights = its cell volumes; empty = tensor product
    std::vector<double> dv_xi, dv_w;
    double R = 0, omega = 0, Tref = 0, mu_ref = 0, Pr = 0;
    int K_inner = 0;
    std::vector<PatchKind> kinds;       // per mesh patch
    std::vector<std::string> rho_types, U_types, T_types;
    std::vector<double> patch_rho, patch_U, patch_T;   // per mesh patch: first face value
    std::vector<double> patch_p;                       // per mesh patch: pressureIn / pressureOut
    std::vector<double> rho0, U0, T0;   // initial cell fields
    // system/controlDict (0 when absent)
    double start_time = 0, end_time = 0, delta_t = 0, write_interval = 0;
    // adjustable time step (src/readTimeControlsExplicit.H:39-46, OpenFOAM's
    // GREAT = 1e15 as the maxDeltaT default)
    bool adjust_time_step = false;
    double max_co = 1.0, max_delta_t = 1.0e15;
};
// vmesh: take the DVs from constant/vMesh instead of Xis/weights
Case read_case(const std::string& dir, bool vmesh = false);

// fv addressing and geometry for dugks_create: internal faces, then the faces
// of the non-empty patches in patch order (empty patches have no fv faces)
struct FlatMesh {
    int32_t n_cells = 0, n_internal = 0, n_boundary = 0, D = 3;
    std::vector<int64_t> owner, neighbour;
    std::vector<double> C, V, Cf, Sf;
    std::vector<int32_t> patch_type, patch_start;   // non-empty patches
    std::vector<int> patch_of;                      // non-empty patch -> mesh patch index
    std::vector<double> rho_b, U_b, T_b, p_b;       // per boundary face
};
// geometry by the library's dugks_mesh_geometry (OpenFOAM primitiveMesh algorithm)
FlatMesh flatten(const Case& c);

// Writes <dir>/<time>/<name> as an OpenFOAM ASCII volume field; patches
// are (name, type, values) with values empty for entries without a value.
void write_vol_field(const std::string& path, const std::string& name, int ncomp, const std::vector<double>& internal,
                     const std::vector<std::pair<std::string, std::pair<std::string, std::vector<double>>>>& patches,
                     const std::string& dims, const std::string& location);

// time directory name as OpenFOAM prints it (general format, 6 digits)
std::string time_name(double t);

}  // namespace dugks_host
