// Pose output in the reference's formats: PDBQT MODEL blocks with the
// "REMARK VINA RESULT" header (unidock/src/lib/vina.cpp:725-748, model.cpp:726-846)
// and SDF records with the "> <Uni-Dock RESULT>" block (vina.cpp:750-770,
// model.cpp:850-866).
#include <cstdio>
#include <iomanip>
#include <sstream>
#include <stdexcept>

#include "ud_model.h"

namespace ud {

// std::fixed with setw(width) and setprecision(prec), as the reference's streams format
static std::string fixed(float v, int width, int prec) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%*.*f", width, prec, (double)v);
    return buf;
}

static void put_coord(std::string& line, std::size_t col, float v) {  // 1-based column, 8 wide
    std::string s = fixed(v, 8, 3);
    if (s.size() != 8) throw std::runtime_error("coordinate does not fit PDBQT columns");
    if (line.size() < col - 1 + 8) line.resize(col - 1 + 8, ' ');
    line.replace(col - 1, 8, s);
}

static std::string vina_remarks(const PoseResult& p, bool ad4) {
    std::ostringstream r;
    r << "REMARK VINA RESULT: " << fixed(p.e, 9, 3) << "  " << fixed(p.lb, 9, 3) << "  " << fixed(p.ub, 9, 3)
      << '\n';
    r << "REMARK INTER + INTRA:    " << fixed(p.total, 12, 3) << "\n";
    r << "REMARK INTER:            " << fixed(p.inter, 12, 3) << "\n";
    r << "REMARK INTRA:            " << fixed(p.intra, 12, 3) << "\n";
    if (ad4) r << "REMARK CONF_INDEPENDENT: " << fixed(p.conf_indep, 12, 3) << "\n";
    r << "REMARK UNBOUND:          " << fixed(p.unbound, 12, 3) << "\n";
    return r.str();
}

static std::string sdf_remarks(const PoseResult& p, bool ad4) {
    std::ostringstream r;
    r << "> <Uni-Dock RESULT> \nENERGY=" << fixed(p.e, 9, 3) << "  LOWER_BOUND=" << fixed(p.lb, 9, 3)
      << "  UPPER_BOUND=" << fixed(p.ub, 9, 3) << '\n';
    r << "INTER + INTRA:    " << fixed(p.total, 12, 3) << "\n";
    r << "INTER:            " << fixed(p.inter, 12, 3) << "\n";
    r << "INTRA:            " << fixed(p.intra, 12, 3) << "\n";
    if (ad4) r << "CONF_INDEPENDENT: " << fixed(p.conf_indep, 12, 3) << "\n";
    r << "UNBOUND:          " << fixed(p.unbound, 12, 3) << "\n";
    r << '\n';
    return r.str();
}

std::string write_pdbqt_models(const Ligand& lig, const std::vector<PoseResult>& poses, bool ad4) {
    std::ostringstream out;
    std::vector<float> xyz(3 * lig.atoms.size());
    for (std::size_t m = 0; m < poses.size(); ++m) {
        ligand_coords(lig, poses[m].pose.data(), xyz.data());
        out << "MODEL " << (m + 1) << '\n';
        out << vina_remarks(poses[m], ad4);
        for (const auto& c : lig.context) {
            if (c.second >= 0) {
                std::string line = c.first;
                put_coord(line, 31, xyz[3 * c.second]);
                put_coord(line, 39, xyz[3 * c.second + 1]);
                put_coord(line, 47, xyz[3 * c.second + 2]);
                out << line << '\n';
            } else {
                out << c.first << '\n';
            }
        }
        out << "ENDMDL\n";
    }
    return out.str();
}

static void put_sdf_coord(std::string& line, std::size_t col, float v) {  // 1-based column, 10 wide
    std::string s = fixed(v, 10, 4);
    if (s.size() != 10) throw std::runtime_error("coordinate does not fit SDF columns");
    if (line.size() < col - 1 + 10) line.resize(col - 1 + 10, ' ');
    line.replace(col - 1, 10, s);
}

// A ligand read from SDF is written back as its own record, each atom line
// with the pose's coordinates (model.cpp:779-785, 822-863): the input lines in
// order ("$$$$" lines were dropped at parse time), then the result block and
// "$$$$".
static std::string write_sdf_context(const Ligand& lig, const std::vector<PoseResult>& poses, bool ad4) {
    std::ostringstream out;
    std::vector<float> xyz(3 * lig.atoms.size());
    for (std::size_t m = 0; m < poses.size(); ++m) {
        ligand_coords(lig, poses[m].pose.data(), xyz.data());
        for (const auto& c : lig.context) {
            if (c.second >= 0) {
                std::string line = c.first;
                put_sdf_coord(line, 1, xyz[3 * c.second]);
                put_sdf_coord(line, 11, xyz[3 * c.second + 1]);
                put_sdf_coord(line, 21, xyz[3 * c.second + 2]);
                out << line << '\n';
            } else {
                out << c.first << '\n';
            }
        }
        out << sdf_remarks(poses[m], ad4);
        out << "$$$$\n";
    }
    return out.str();
}

// The ligand's input record at one pose with no result block: an SDF
// ligand in SDF columns, a PDBQT one in PDBQT columns (model.h:125-144,
// write_structure / write_sdf_structure).
std::string write_structure(const Ligand& lig, const float* pose) {
    std::vector<float> xyz(3 * lig.atoms.size());
    ligand_coords(lig, pose, xyz.data());
    std::ostringstream out;
    for (const auto& c : lig.context) {
        if (c.second < 0) {
            out << c.first << '\n';
            continue;
        }
        std::string line = c.first;
        const float* x = &xyz[3 * c.second];
        if (lig.sdf) {
            put_sdf_coord(line, 1, x[0]);
            put_sdf_coord(line, 11, x[1]);
            put_sdf_coord(line, 21, x[2]);
        } else {
            put_coord(line, 31, x[0]);
            put_coord(line, 39, x[1]);
            put_coord(line, 47, x[2]);
        }
        out << line << '\n';
    }
    return out.str();
}

std::string write_sdf_models(const Ligand& lig, const std::vector<PoseResult>& poses, bool ad4) {
    if (lig.sdf) return write_sdf_context(lig, poses, ad4);
    // PDBQT input is written as a minimal V2000 block of its atoms.
    std::ostringstream out;
    std::vector<float> xyz(3 * lig.atoms.size());
    static const char* el_name[] = {"H", "C", "N", "O", "S", "P", "F", "Cl", "Br", "I", "Si", "At", "X", "X"};
    for (std::size_t m = 0; m < poses.size(); ++m) {
        ligand_coords(lig, poses[m].pose.data(), xyz.data());
        out << (lig.name.empty() ? "ligand" : lig.name) << "\n  unidock_b200\n\n";
        int nb = 0;
        for (auto& a : lig.atoms) nb += (int)a.bonds.size();
        nb /= 2;
        char buf[128];
        std::snprintf(buf, sizeof buf, "%3d%3d  0  0  0  0  0  0  0  0999 V2000\n", (int)lig.atoms.size(), nb);
        out << buf;
        for (std::size_t i = 0; i < lig.atoms.size(); ++i) {
            int el = lig.atoms[i].el;
            const char* nm = (el >= 0 && el < 14) ? el_name[el] : "X";
            std::snprintf(buf, sizeof buf, "%10.4f%10.4f%10.4f %-3s 0  0  0  0  0  0  0  0  0  0  0  0\n",
                          xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], nm);
            out << buf;
        }
        for (std::size_t i = 0; i < lig.atoms.size(); ++i)
            for (int j : lig.atoms[i].bonds)
                if ((int)i < j) {
                    std::snprintf(buf, sizeof buf, "%3d%3d  1  0\n", (int)i + 1, j + 1);
                    out << buf;
                }
        out << "M  END\n";
        out << sdf_remarks(poses[m], ad4);
        out << "$$$$\n";
    }
    return out.str();
}

}  // namespace ud
