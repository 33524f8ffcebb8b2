// Edge cases of wf::load_obj (the reference's OBJ contract, WVM/src/obj_loader.cpp:49-186): line
// endings, tabs and comments, face tokens with '/', many-cornered faces, and the error messages with
// their 1-based line numbers. Built against libwf_core.so and run by tests/test_obj_loader.py; prints
// one line per failed check and exits 1 if any failed.
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include "wf/scene.hpp"

namespace {

int g_failed = 0;

void expect(bool ok, const std::string& what) {
    if (!ok) {
        std::printf("FAILED: %s\n", what.c_str());
        ++g_failed;
    }
}

std::string write(const std::string& dir, const std::string& name, const std::string& text) {
    const std::string path = dir + "/" + name;
    std::ofstream(path, std::ios::binary) << text;
    return path;
}

std::string error_of(const std::string& path) {
    try {
        wf::load_obj(path, 16, 9);
    } catch (const std::runtime_error& e) {
        return e.what();
    }
    return "";
}

bool contains(const std::string& s, const std::string& part) { return s.find(part) != std::string::npos; }

}  // namespace

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    const std::string dir = argv[1];

    {  // CRLF, tabs, trailing comments, no final newline
        const wf::Scene s = wf::load_obj(write(dir, "crlf.obj", "v 0 0 0\r\nv\t1 0 0 # x\r\n\r\nv 0 1 0\r\nf 1 2 3"), 16, 9);
        expect(s.vertices.size() == 3 && s.triangles.size() == 1, "CRLF / tabs / comments / no final newline");
        expect(s.vertices[1].x == 1.0f && s.vertices[2].y == 1.0f, "vertex values");
    }
    {  // face tokens with texture / normal indices
        const wf::Scene s = wf::load_obj(write(dir, "slash.obj", "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1/1/1 2//2 3/3 4\n"), 16, 9);
        expect(s.triangles.size() == 2, "quad with slashed indices gives 2 triangles");
        expect(s.triangles[1].i0 == 0 && s.triangles[1].i1 == 2 && s.triangles[1].i2 == 3, "fan triangulation order");
    }
    {  // a face with more corners than the tokenizer's first guess
        std::string text;
        for (int k = 0; k < 100; ++k) text += "v " + std::to_string(k) + " " + std::to_string(k * k % 7) + " 0\n";
        text += "f";
        for (int k = 1; k <= 100; ++k) text += " " + std::to_string(k);
        text += "\n";
        const wf::Scene s = wf::load_obj(write(dir, "big.obj", text), 16, 9);
        expect(s.triangles.size() == 98, "100-corner face gives 98 triangles");
        expect(s.triangles[97].i0 == 0 && s.triangles[97].i1 == 98 && s.triangles[97].i2 == 99, "last fan triangle");
    }
    // errors, with the 1-based line number of the offending line
    expect(contains(error_of(write(dir, "e1.obj", "v 1.5x 0 0\nf 1 1 1\n")), "line 1: malformed vertex coordinate"),
           "malformed coordinate");
    expect(contains(error_of(write(dir, "e2.obj", "# c\n\nv 0 0\n")), "line 3: a vertex needs exactly 3 coordinates"),
           "vertex arity, comment and blank lines counted");
    expect(contains(error_of(write(dir, "e3.obj", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 /2 3\n")),
                    "line 4: malformed face index '/2'"),
           "face token without a vertex index");
    expect(contains(error_of(write(dir, "e4.obj", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n")), "face index 4 outside 1..3"),
           "face index out of range");
    expect(contains(error_of(write(dir, "e5.obj", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 99999999999999999999\n")),
                    "malformed face index"),
           "face index overflow");
    expect(contains(error_of(write(dir, "e6.obj", "v 0 0 0\nv 1 0 0\nf 1 2\n")), "line 3: a face needs at least 3 indices"),
           "face arity");
    expect(contains(error_of(write(dir, "e7.obj", "")), "no faces"), "empty file");
    expect(contains(error_of(dir + "/missing.obj"), "cannot open"), "missing file");
    // Large files (parsed in chunks of lines on several threads): same arrays, and the first error in
    // file order with its line number and the vertex count seen before it.
    {
        const int nv = 400000;  // about 9 MB of text: several chunks
        std::string text = "# big\n";
        for (int k = 0; k < nv; ++k) {
            text += "v " + std::to_string(k % 1000) + ".5 " + std::to_string(k / 1000) + " -" + std::to_string(k % 7) + "\n";
            if (k >= 2 && k % 3 == 2) text += "f " + std::to_string(k - 1) + "/1 " + std::to_string(k) + " " + std::to_string(k + 1) + "\r\n";
        }
        const wf::Scene s = wf::load_obj(write(dir, "big_ok.obj", text), 16, 9);
        bool same = s.vertices.size() == (size_t)nv && s.triangles.size() == (size_t)((nv - 2 + 2) / 3);
        for (int k = 0; same && k < nv; k += 997)
            same = s.vertices[k].x == (float)(k % 1000) + 0.5f && s.vertices[k].y == (float)(k / 1000) &&
                   s.vertices[k].z == -(float)(k % 7);
        for (size_t t = 0; same && t < s.triangles.size(); t += 991) {
            const int k = 2 + 3 * (int)t;
            same = s.triangles[t].i0 == k - 2 && s.triangles[t].i1 == k - 1 && s.triangles[t].i2 == k;
        }
        expect(same, "large file: vertices and triangles in file order");
        // a face late in the file that names a vertex defined after it; and an earlier malformed vertex
        const std::string late = text + "f 1 2 " + std::to_string(nv + 1) + "\nv 0 0 0\n";
        const int late_line = 1 + nv + (nv - 1) / 3 + 1;
        expect(contains(error_of(write(dir, "big_late.obj", late)),
                        "line " + std::to_string(late_line) + ": face index " + std::to_string(nv + 1) + " outside 1.." +
                            std::to_string(nv)),
               "large file: face index past the vertices seen so far");
        std::string two = text;
        two.insert(two.size() / 4, "\nv 1 2\n");  // an error in an early chunk ...
        two += "f 0 1 2\n";                       // ... wins over one in the last chunk
        const std::string e2 = error_of(write(dir, "big_two.obj", two));
        expect(contains(e2, "a vertex needs exactly 3 coordinates") && !contains(e2, "malformed face index"),
               "large file: the first error in file order is reported");
    }
    std::printf("obj loader checks: %d failed\n", g_failed);
    return g_failed == 0 ? 0 : 1;
}
