// lpg_veg.cpp -- VEG volume-mesh files: read_veg and write_veg of the reference's mesh I/O
// (src/core/mesh/io/veg.cpp), written here from the format's grammar.
//
// Grammar (one record per line; fields separated by spaces, tabs or commas):
//
//   file       := { blank | comment | directive | record }
//   comment    := '#' anything
//   directive  := '*' keyword { field }
//   *INCLUDE p    the lines of file p (relative to the including file) in place; a file that
//                 includes itself, directly or through others, is an error
//   *VERTICES     header "count 3 ..." then `count` records "id x y z ..."; ids start at 0 or 1
//                 and increase by one (the first id fixes the base of every vertex reference)
//   *ELEMENTS     a type record (TET or CUBIC, blanks inside ignored), header "count width ...",
//                 then `count` records "id v_1 .. v_width ..." of vertex references
//   *other        material, set and region directives: their records are skipped
//
// A file holds one *VERTICES section and, after it, one *ELEMENTS section. Problems with the
// file or its format raise LPG_EIO (the reference's std::runtime_error), with the file and line
// where they were found; a file that parses into an invalid mesh (non-finite coordinates,
// repeated vertices in a cell) raises LPG_EINVAL (its std::invalid_argument).

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <memory>
#include <string>
#include <string_view>
#include <vector>

#include "lpg_internal.h"

namespace lpg {
namespace fs = std::filesystem;

namespace {

bool blank(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }
bool separator(char c) { return blank(c) || c == ','; }

std::string_view trim(std::string_view s) {
    while (!s.empty() && blank(s.front())) s.remove_prefix(1);
    while (!s.empty() && blank(s.back())) s.remove_suffix(1);
    return s;
}

// A meaningful line and the place it was read from.
struct Line {
    std::string text;
    std::string where; // "file:line"
    bool directive() const { return !text.empty() && text[0] == '*'; }
    // The directive's keyword: the letters after '*' up to the first separator.
    std::string_view keyword() const {
        std::string_view t(text);
        t.remove_prefix(1);
        size_t n = 0;
        while (n < t.size() && !separator(t[n])) ++n;
        return t.substr(0, n);
    }
};

// Lines of a VEG file with *INCLUDE directives followed in place. Blank and comment lines are
// dropped. The open files form a stack; a file already on it may not be opened again.
class LineSource {
public:
    explicit LineSource(const fs::path& root) { open(root, ""); }

    // The next meaningful line; false once the root file is exhausted.
    bool next(Line& out) {
        while (!files_.empty()) {
            File& f = *files_.back();
            std::string raw;
            if (!std::getline(f.in, raw)) {
                if (f.in.bad()) fail(LPG_EIO, "VEG: read error in " + f.path.string());
                files_.pop_back();
                continue;
            }
            ++f.line;
            const std::string_view t = trim(raw);
            if (t.empty() || t[0] == '#') continue;
            const std::string where = f.path.string() + ":" + std::to_string(f.line);
            if (t.substr(0, 8) == "*INCLUDE" && (t.size() == 8 || blank(t[8]))) {
                const std::string_view target = trim(t.substr(8));
                if (target.empty()) fail(LPG_EIO, "VEG " + where + ": *INCLUDE names no file");
                open(f.path.parent_path() / std::string(target), where);
                continue;
            }
            out.text.assign(t);
            out.where = where;
            return true;
        }
        return false;
    }

private:
    struct File {
        std::ifstream in;
        fs::path path, key;
        long line = 0;
    };
    std::vector<std::unique_ptr<File>> files_;

    void open(const fs::path& path, const std::string& from) {
        std::error_code ec;
        fs::path key = fs::weakly_canonical(path, ec);
        if (ec) key = path;
        for (const auto& f : files_)
            if (f->key == key) fail(LPG_EIO, "VEG " + from + ": include cycle: " + path.string() + " is already being read");
        auto f = std::make_unique<File>();
        f->in.open(path, std::ios::binary);
        if (!f->in) fail(LPG_EIO, "VEG: cannot open " + path.string() + (from.empty() ? "" : " (included at " + from + ")"));
        f->path = path;
        f->key = key;
        files_.push_back(std::move(f));
    }
};

// The numeric fields of a record, each parsed in full (std::from_chars).
template <class T> std::vector<T> numbers(const Line& line) {
    std::vector<T> out;
    const char* p = line.text.data();
    const char* end = p + line.text.size();
    while (true) {
        while (p < end && separator(*p)) ++p;
        if (p == end) break;
        const char* q = p;
        while (q < end && !separator(*q)) ++q;
        T v{};
        const char* s = (*p == '+' && q - p > 1) ? p + 1 : p; // from_chars takes no leading '+'
        const auto r = std::from_chars(s, q, v);
        if (r.ec != std::errc() || r.ptr != q)
            fail(LPG_EIO, "VEG " + line.where + ": '" + std::string(p, q) + "' is not a number (record '" + line.text + "')");
        out.push_back(v);
        p = q;
    }
    return out;
}

// Reads a VEG mesh from a line source: a small state machine over the directives.
class VegParser {
public:
    VegParser(const fs::path& root, VegMesh& mesh) : src_(root), mesh_(mesh), root_(root.string()) {}

    void run() {
        mesh_ = VegMesh{};
        Line line;
        bool have = src_.next(line);
        while (have) {
            if (!line.directive()) { // a record of a skipped section
                have = src_.next(line);
                continue;
            }
            const std::string_view kw = line.keyword();
            if (kw == "VERTICES")
                vertices(line);
            else if (kw == "ELEMENTS")
                elements(line);
            have = src_.next(line);
        }
        if (!seen_vertices_) fail(LPG_EIO, "VEG " + root_ + ": the file has no *VERTICES section");
        if (mesh_.width == 0) fail(LPG_EIO, "VEG " + root_ + ": the file has no *ELEMENTS section");
    }

private:
    LineSource src_;
    VegMesh& mesh_;
    std::string root_;
    bool seen_vertices_ = false;
    long base_ = 1;

    // The next line, which must be a record of the section `what` opened at `at`.
    Line record(const Line& at, const char* what) {
        Line r;
        if (!src_.next(r)) fail(LPG_EIO, "VEG " + at.where + ": the file ends inside the " + what);
        if (r.directive()) fail(LPG_EIO, "VEG " + r.where + ": expected the " + std::string(what) + ", found '" + r.text + "'");
        return r;
    }

    void vertices(const Line& at) {
        if (seen_vertices_) fail(LPG_EIO, "VEG " + at.where + ": a second *VERTICES section");
        seen_vertices_ = true;
        const Line h = record(at, "vertex header");
        const std::vector<long> head = numbers<long>(h);
        if (head.size() < 2 || head[0] < 0 || head[0] > (1L << 31) - 1 || head[1] != 3)
            fail(LPG_EIO, "VEG " + h.where + ": the vertex header must read '<count> 3 ...', got '" + h.text + "'");
        const long n = head[0];
        mesh_.positions.reserve(3 * static_cast<size_t>(std::min(n, 1L << 20))); // the count is not trusted
        for (long k = 0; k < n; ++k) {
            const Line r = record(at, "vertex records");
            const std::vector<double> v = numbers<double>(r);
            if (v.size() < 4) fail(LPG_EIO, "VEG " + r.where + ": a vertex record needs an id and three coordinates");
            if (k == 0) base_ = v[0] == 0.0 ? 0 : 1;
            if (v[0] != static_cast<double>(k + base_))
                fail(LPG_EIO, "VEG " + r.where + ": vertex id " + std::to_string(v[0]) + " where " +
                                  std::to_string(k + base_) + " was expected (ids run consecutively)");
            mesh_.positions.push_back(v[1]);
            mesh_.positions.push_back(v[2]);
            mesh_.positions.push_back(v[3]);
        }
        mesh_.num_vertices = static_cast<int>(n);
    }

    void elements(const Line& at) {
        if (!seen_vertices_) fail(LPG_EIO, "VEG " + at.where + ": *ELEMENTS before any *VERTICES section");
        if (mesh_.width != 0) fail(LPG_EIO, "VEG " + at.where + ": a second *ELEMENTS section");
        const Line t = record(at, "element type");
        std::string type;
        for (char c : t.text)
            if (!blank(c)) type.push_back(c);
        const int width = type == "TET" ? 4 : type == "CUBIC" ? 8 : 0;
        if (width == 0) fail(LPG_EIO, "VEG " + t.where + ": element type '" + type + "' is neither TET nor CUBIC");
        const Line h = record(at, "element header");
        const std::vector<long> head = numbers<long>(h);
        if (head.empty() || head[0] < 0 || head[0] > (1L << 31) - 1)
            fail(LPG_EIO, "VEG " + h.where + ": the element header must start with a non-negative count");
        if (head.size() < 2 || head[1] != width)
            fail(LPG_EIO, "VEG " + h.where + ": " + type + " elements have " + std::to_string(width) +
                              " vertices, the header says '" + h.text + "'");
        const long m = head[0];
        mesh_.cells.reserve(static_cast<size_t>(std::min(m, 1L << 20)) * width);
        for (long k = 0; k < m; ++k) {
            const Line r = record(at, "element records");
            const std::vector<long> v = numbers<long>(r);
            if (static_cast<long>(v.size()) < width + 1)
                fail(LPG_EIO, "VEG " + r.where + ": an element record needs an id and " + std::to_string(width) +
                                  " vertex references");
            for (int a = 1; a <= width; ++a) {
                const long id = v[a] - base_;
                if (id < 0 || id >= mesh_.num_vertices)
                    fail(LPG_EIO, "VEG " + r.where + ": vertex reference " + std::to_string(v[a]) +
                                      " is not one of the file's vertices");
                mesh_.cells.push_back(static_cast<int32_t>(id));
            }
        }
        mesh_.width = width;
    }
};

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
    VegParser(fs::path(file), mesh).run();
    validate_volume_mesh(mesh.num_vertices, mesh.positions, mesh.width, mesh.cells);
}

void write_veg(const std::string& file, int V, const double* positions, int T, int width, const int32_t* cells) {
    if (V < 0 || T < 0 || (width != 4 && width != 8)) fail(LPG_EINVAL, "write_veg: a tet (4) or hex (8) volume mesh is required");
    std::vector<double> pos(positions, positions + 3 * static_cast<size_t>(V));
    std::vector<int32_t> cl(cells, cells + static_cast<size_t>(width) * T);
    validate_volume_mesh(V, pos, width, cl);
    std::FILE* f = std::fopen(file.c_str(), "w");
    if (!f) fail(LPG_EIO, "VEG: cannot open " + file + " for writing");
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
    if (!ok) fail(LPG_EIO, "VEG: writing " + file + " failed");
}

} // namespace lpg
