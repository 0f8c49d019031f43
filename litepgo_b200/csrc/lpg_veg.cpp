// lpg_veg.cpp -- VEG volume-mesh files (the reference's src/core/mesh/io/veg.cpp, read_veg and
// write_veg): the text format of libpgo/Vega with a *VERTICES section ("n 3 ..." then one
// "id x y z" line per vertex, ids consecutive from 0 or 1) and one *ELEMENTS section (a type
// line, TET or CUBIC, then "m width ..." and one "id v1 .. v_width" line per element, vertex ids
// in the vertices' base). Blank lines and lines starting with '#' are skipped, "*INCLUDE name"
// splices another file (relative to the including one; cycles are an error) and every other
// record is ignored. Fields may be separated by spaces, tabs or commas.
//
// File and format problems raise LPG_EIO (the reference's std::runtime_error); a mesh that
// parses but is not a valid mesh (non-finite coordinates, repeated vertices in a cell) raises
// LPG_EINVAL (its std::invalid_argument).

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <limits>
#include <string>
#include <type_traits>
#include <vector>

#include "lpg_internal.h"

namespace lpg {
namespace fs = std::filesystem;

namespace {

[[noreturn]] void io_fail(const std::string& what) { fail(LPG_EIO, what); }

std::string strip(const std::string& s) {
    const char* ws = " \t\r\n";
    const size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) return {};
    return s.substr(a, s.find_last_not_of(ws) - a + 1);
}

// The meaningful lines of a file, *INCLUDE files spliced in place. `chain` holds the files being
// read around this one.
void load_lines(const fs::path& path, std::vector<fs::path>& chain, std::vector<std::string>& out) {
    const fs::path key = fs::weakly_canonical(path);
    for (const fs::path& p : chain)
        if (p == key) io_fail("veg *INCLUDE cycle through " + path.string());
    std::ifstream in(path, std::ios::binary);
    if (!in) io_fail("Failed to open veg file: " + path.string());
    chain.push_back(key);
    std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    if (in.bad()) io_fail("Failed reading VEG: " + path.string());
    size_t pos = 0;
    while (pos < text.size()) {
        size_t eol = text.find('\n', pos);
        if (eol == std::string::npos) eol = text.size();
        size_t a = pos, b = eol;
        while (a < b && (text[a] == ' ' || text[a] == '\t' || text[a] == '\r')) ++a;
        while (b > a && (text[b - 1] == ' ' || text[b - 1] == '\t' || text[b - 1] == '\r')) --b;
        pos = eol + 1;
        if (a == b || text[a] == '#') continue;
        std::string line(text, a, b - a);
        if (line.compare(0, 9, "*INCLUDE ") == 0) {
            load_lines(path.parent_path() / strip(line.substr(9)), chain, out);
            continue;
        }
        out.push_back(std::move(line));
    }
    chain.pop_back();
}

// Splits a record into fields (space, tab or comma separated) and parses each completely as a
// number; false if a field is not one.
template <class T> bool fields(const std::string& line, std::vector<T>& out) {
    out.clear();
    size_t i = 0;
    const size_t n = line.size();
    auto sep = [](char c) { return c == ' ' || c == '\t' || c == ',' || c == '\r' || c == '\n'; };
    while (i < n) {
        while (i < n && sep(line[i])) ++i;
        if (i >= n) break;
        size_t j = i;
        while (j < n && !sep(line[j])) ++j;
        // Parse in place; the number must end exactly where the field ends.
        const char* beg = line.c_str() + i;
        char* end = nullptr;
        if constexpr (std::is_same<T, double>::value) {
            const double v = std::strtod(beg, &end);
            if (end != line.c_str() + j) return false;
            out.push_back(v);
        } else {
            const long long v = std::strtoll(beg, &end, 10);
            if (end != line.c_str() + j || v < std::numeric_limits<int>::min() || v > std::numeric_limits<int>::max())
                return false;
            out.push_back(static_cast<T>(v));
        }
        i = j;
    }
    return true;
}

template <class T> std::vector<T> record(const std::string& line) {
    std::vector<T> v;
    if (!fields(line, v)) io_fail("Malformed VEG numeric record: " + line);
    return v;
}

std::string no_space(const std::string& s) {
    std::string r;
    for (char c : s)
        if (c != ' ' && c != '\t' && c != '\r' && c != '\n') r.push_back(c);
    return r;
}

} // namespace

void validate_volume_mesh(int V, const std::vector<double>& positions, int width, const std::vector<int32_t>& cells) {
    if (positions.size() != 3 * static_cast<size_t>(V)) fail(LPG_EINVAL, "MeshData requires three finite coordinates per vertex");
    for (double x : positions)
        if (!std::isfinite(x)) fail(LPG_EINVAL, "MeshData requires three finite coordinates per vertex");
    const size_t T = width > 0 ? cells.size() / static_cast<size_t>(width) : 0;
    for (size_t e = 0; e < T; ++e)
        for (int a = 0; a < width; ++a) {
            const int32_t v = cells[e * width + a];
            if (v < 0 || v >= V)
                fail(LPG_EINVAL, "MeshTopology cell " + std::to_string(e) + " has vertex indices outside [0, num_vertices)");
            for (int b = 0; b < a; ++b)
                if (cells[e * width + b] == v)
                    fail(LPG_EINVAL, "MeshTopology cell " + std::to_string(e) + " must contain distinct vertices");
        }
}

void read_veg(const std::string& file, VegMesh& mesh) {
    const fs::path path(file);
    std::vector<std::string> lines;
    std::vector<fs::path> chain;
    load_lines(path, chain, lines);
    mesh = VegMesh{};
    const std::string where = " in " + path.string();
    int base = 1; // 1-based vertex ids unless the first one is 0
    bool have_vertices = false;
    size_t i = 0;
    while (i < lines.size()) {
        const std::string& line = lines[i];
        if (line.compare(0, 9, "*VERTICES") == 0) {
            if (have_vertices) io_fail("Duplicate *VERTICES section" + where);
            have_vertices = true;
            if (++i >= lines.size()) io_fail("Missing *VERTICES header" + where);
            const std::vector<int> head = record<int>(lines[i++]);
            if (head.size() < 2 || head[0] < 0 || head[1] != 3) io_fail("Invalid 3D vertex header" + where);
            const size_t n = static_cast<size_t>(head[0]);
            if (n > lines.size() - i) io_fail("Truncated vertex data" + where);
            mesh.positions.reserve(3 * n);
            for (size_t row = 0; row < n; ++row, ++i) {
                const std::vector<double> v = record<double>(lines[i]);
                if (v.size() < 4) io_fail("Malformed vertex line" + where + ": " + lines[i]);
                if (row == 0 && v[0] == 0) base = 0;
                if (v[0] != static_cast<double>(row) + base) io_fail("Vertex IDs must be consecutive" + where);
                mesh.positions.insert(mesh.positions.end(), {v[1], v[2], v[3]});
            }
            mesh.num_vertices = static_cast<int>(n);
            continue;
        }
        if (line.compare(0, 9, "*ELEMENTS") == 0) {
            if (!have_vertices || mesh.width != 0)
                io_fail("Expected one *VERTICES section followed by one *ELEMENTS section" + where);
            if (++i >= lines.size()) io_fail("Missing element type" + where);
            const std::string type = no_space(lines[i++]);
            if (type == "TET")
                mesh.width = 4;
            else if (type == "CUBIC")
                mesh.width = 8;
            else
                io_fail("Unsupported element type" + where + ": " + type);
            if (i >= lines.size()) io_fail("Missing element count" + where);
            const std::vector<int> head = record<int>(lines[i++]);
            if (head.empty() || head[0] < 0) io_fail("Invalid element count" + where);
            const size_t m = static_cast<size_t>(head[0]);
            if (m > lines.size() - i) io_fail("Truncated element data" + where);
            if (head.size() < 2 || head[1] != mesh.width) io_fail("Element width does not match its type" + where);
            mesh.cells.reserve(m * static_cast<size_t>(mesh.width));
            for (size_t row = 0; row < m; ++row, ++i) {
                const std::vector<int> v = record<int>(lines[i]);
                if (static_cast<int>(v.size()) < mesh.width + 1) io_fail("Malformed element line" + where + ": " + lines[i]);
                for (int a = 1; a <= mesh.width; ++a) {
                    const long long id = static_cast<long long>(v[a]) - base;
                    if (id < 0 || id >= mesh.num_vertices) io_fail("Element vertex index out of range" + where);
                    mesh.cells.push_back(static_cast<int32_t>(id));
                }
            }
            continue;
        }
        ++i; // materials, sets, regions and other records carry no geometry
    }
    if (mesh.width == 0) io_fail("No *ELEMENTS section found" + where);
    validate_volume_mesh(mesh.num_vertices, mesh.positions, mesh.width, mesh.cells);
}

void write_veg(const std::string& file, int V, const double* positions, int T, int width, const int32_t* cells) {
    if (V < 0 || T < 0 || (width != 4 && width != 8)) fail(LPG_EINVAL, "write_veg: a tet (4) or hex (8) volume mesh is required");
    std::vector<double> pos(positions, positions + 3 * static_cast<size_t>(V));
    std::vector<int32_t> cl(cells, cells + static_cast<size_t>(width) * T);
    validate_volume_mesh(V, pos, width, cl);
    std::FILE* f = std::fopen(file.c_str(), "w");
    if (!f) io_fail("Cannot write VEG: " + file);
    bool ok = std::fprintf(f, "*VERTICES\n%d 3 0 0\n", V) > 0;
    for (int v = 0; v < V && ok; ++v)
        ok = std::fprintf(f, "%d %.17g %.17g %.17g\n", v + 1, pos[3 * size_t(v)], pos[3 * size_t(v) + 1],
                          pos[3 * size_t(v) + 2]) > 0;
    ok = ok && std::fprintf(f, "*ELEMENTS\n%s\n%d %d 0\n", width == 4 ? "TET" : "CUBIC", T, width) > 0;
    for (int e = 0; e < T && ok; ++e) {
        ok = std::fprintf(f, "%d", e + 1) > 0;
        for (int a = 0; a < width && ok; ++a) ok = std::fprintf(f, " %d", cl[size_t(e) * width + a] + 1) > 0;
        ok = ok && std::fputc('\n', f) != EOF;
    }
    if (std::fclose(f) != 0) ok = false;
    if (!ok) io_fail("Failed writing VEG: " + file);
}

} // namespace lpg
