// Drop-in for the reference verifier gpart_verify_csr (tools/verify_csr.cpp):
//   indptr indices k partition binary|text [--symmetric]
// prints one JSON line and exits 0 (capacity ok), 1 (violated) or 2 (error).
// Without extensions the capacity is the reference's n*103/(100k) with unit
// loads.  Extensions for weighted inputs: --vertex-weights f --edge-weights f
// (raw uint32 files) and --epsilon e (capacity floor(total*e/k)).
#include "gpart_b200.h"

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {
void check(gp_status s) {
    if (s != GP_OK) throw std::runtime_error(gp_last_error());
}
template <class T>
std::vector<T> read_raw(const std::string& path) {
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) throw std::runtime_error("invalid input file");
    const auto bytes = static_cast<size_t>(in.tellg());
    if (bytes % sizeof(T)) throw std::runtime_error("invalid input file");
    std::vector<T> v(bytes / sizeof(T));
    in.seekg(0);
    if (bytes) in.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(bytes));
    return v;
}
}  // namespace

int main(int argc, char** argv) {
    try {
        std::vector<std::string> args(argv + 1, argv + argc);
        bool symmetric = false;
        std::string vw_path, ew_path;
        double epsilon = 0.0;
        std::vector<std::string> pos;
        for (size_t i = 0; i < args.size(); ++i) {
            if (args[i] == "--symmetric") symmetric = true;
            else if (args[i] == "--vertex-weights" && i + 1 < args.size()) vw_path = args[++i];
            else if (args[i] == "--edge-weights" && i + 1 < args.size()) ew_path = args[++i];
            else if (args[i] == "--epsilon" && i + 1 < args.size()) epsilon = std::stod(args[++i]);
            else if (args[i].rfind("--", 0) == 0) throw std::runtime_error("invalid flag");
            else pos.push_back(args[i]);
        }
        if (pos.size() != 5) throw std::runtime_error("usage: indptr indices k partition binary|text [--symmetric]");
        const int k = std::stoi(pos[2]);
        if (k < 2 || k > 128) throw std::runtime_error("invalid k");
        int64_t n = 0, m = 0;
        check(gp_read_csr_int64(pos[0].c_str(), pos[1].c_str(), &n, &m, nullptr, nullptr));
        std::vector<int32_t> off(static_cast<size_t>(n + 1)), nbr(static_cast<size_t>(m));
        check(gp_read_csr_int64(pos[0].c_str(), pos[1].c_str(), &n, &m, off.data(), nbr.data()));
        std::vector<int32_t> labels;
        if (pos[4] == "binary") {
            labels = read_raw<int32_t>(pos[3]);
            if (static_cast<int64_t>(labels.size()) != n) throw std::runtime_error("partition length mismatch");
        } else if (pos[4] == "text") {
            std::ifstream in(pos[3]);
            int64_t label;
            if (!in) throw std::runtime_error("cannot read partition");
            while (in >> label) {
                if (label < 0 || label >= k) throw std::runtime_error("invalid label");
                labels.push_back(static_cast<int32_t>(label));
            }
            if (!in.eof() || static_cast<int64_t>(labels.size()) != n) throw std::runtime_error("invalid text partition");
        } else throw std::runtime_error("invalid partition format");
        std::vector<uint32_t> vw, ew;
        if (!vw_path.empty()) vw = read_raw<uint32_t>(vw_path);
        if (!ew_path.empty()) ew = read_raw<uint32_t>(ew_path);
        if ((!vw.empty() && static_cast<int64_t>(vw.size()) != n) || (!ew.empty() && static_cast<int64_t>(ew.size()) != m))
            throw std::runtime_error("weight length mismatch");
        const gp_csr g{n, m, off.data(), nbr.data(), vw.empty() ? nullptr : vw.data(), ew.empty() ? nullptr : ew.data()};
        const bool extended = !vw.empty() || !ew.empty() || epsilon > 0.0;
        std::vector<char> json(256 + 24 * static_cast<size_t>(k));
        uint64_t cut = 0;
        int32_t ok = 0;
        std::vector<uint64_t> loads(static_cast<size_t>(k));
        check(gp_verify(&g, labels.data(), k, extended ? (epsilon > 0.0 ? epsilon : 1.03) : 1.03, symmetric, &cut,
                        loads.data(), &ok, json.data(), json.size()));
        if (!extended) {
            // The reference's integer capacity n*103/(100k) with unit loads.
            uint64_t maximum = 0;
            for (auto l : loads) maximum = l > maximum ? l : maximum;
            const uint64_t capacity = static_cast<uint64_t>(n) * 103 / (100 * static_cast<uint64_t>(k));
            std::string text(json.data());
            const auto a = text.find("\"capacity\":");
            if (a != std::string::npos) text = text.substr(0, a);
            ok = maximum <= capacity;
            text += "\"capacity\":" + std::to_string(capacity) + ",\"capacity_ok\":" + (ok ? "true" : "false") + "}";
            std::cout << text << '\n';
        } else {
            std::cout << json.data() << '\n';
        }
        return ok ? 0 : 1;
    } catch (const std::exception& e) {
        std::cerr << e.what() << '\n';
        return 2;
    }
}
