// ljcell_driver.cpp -- command-line driver with the reference's sweep and CSV.
//
// Mirrors main() of the reference's cell-grid benchmark (cudaLJ.cu:701-792):
// the uniform sweep (box 1, boxDiv = 2..32 doubling, N = boxDiv^3 .. 32 boxDiv^3
// doubling, 5 loops) or, with -gs / --gensurface, the sphere-surface sweep
// (cudaLJ.cu:716-745), each point run through ljcell::executeSimulation, and
// a CSV with the reference's columns (cudaLJ.cu:779-788) written to
// results[-surface]-<date>.csv so existing plotting reads it unchanged.
// Extra flags (not in the reference): --max-box-div D, --loops L, --out FILE.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <ctime>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "ljcell.hpp"

namespace {

struct ResultFrame {
    int nbParticles;
    unsigned long long nbInteractions;
    int nbLoops;
    int boxDiv;
    std::vector<ljcell::AResult> results;
};

std::string default_filename(bool gensurface) {
    std::time_t now = std::chrono::system_clock::to_time_t(std::chrono::system_clock::now());
    char buffer[80];
    std::strftime(buffer, sizeof(buffer), "%Y%m%d-%H%M%S", std::localtime(&now));
    return std::string("results") + (gensurface ? "-surface" : "") + "-" + buffer + ".csv";
}

}  // namespace

int main(int argc, char** argv) {
    bool gensurface = false;
    int maxBoxDiv = -1, loops = 5;
    std::string out;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-gs" || a == "--gensurface") gensurface = true;
        else if (a == "--max-box-div" && i + 1 < argc) maxBoxDiv = std::stoi(argv[++i]);
        else if (a == "--loops" && i + 1 < argc) loops = std::stoi(argv[++i]);
        else if (a == "--out" && i + 1 < argc) out = argv[++i];
        else {
            std::cerr << "usage: " << argv[0] << " [-gs|--gensurface] [--max-box-div D] [--loops L] [--out FILE]\n";
            return 2;
        }
    }
    const int MaxParticlesPerCell = 32;
    std::vector<ResultFrame> all;
    try {
        if (gensurface) {
            const int MaxBoxDiv = maxBoxDiv > 0 ? maxBoxDiv : 128;
            for (int boxDiv = 2; boxDiv <= MaxBoxDiv; boxDiv *= 2) {
                const int nbBoxes = boxDiv * boxDiv * boxDiv;
                for (int n = nbBoxes; n <= nbBoxes * MaxParticlesPerCell; n *= 2) {
                    const double ppc = double(n) / double(nbBoxes);
                    const double coef = 1. - ((2 * 9 * ppc) / n);
                    const double sphereRadius = std::acos(std::min(1.0, std::max(-1.0, coef)));
                    const float boxWidth = std::ceil(2.0 / sphereRadius) * sphereRadius;
                    const int gridDim = static_cast<int>(boxWidth / sphereRadius);
                    const float cellWidth = boxWidth / gridDim;
                    auto [nb, res] = ljcell::executeSimulation<float>(n, loops, boxWidth, cellWidth, false, true);
                    all.push_back(ResultFrame{n, nb, loops, boxDiv, std::move(res)});
                }
            }
        } else {
            const int MaxBoxDiv = maxBoxDiv > 0 ? maxBoxDiv : 32;
            for (int boxDiv = 2; boxDiv <= MaxBoxDiv; boxDiv *= 2) {
                const float cellWidth = 1.0f / boxDiv;
                const int nbBoxes = boxDiv * boxDiv * boxDiv;
                for (int n = nbBoxes; n <= nbBoxes * MaxParticlesPerCell; n *= 2) {
                    auto [nb, res] = ljcell::executeSimulation<float>(n, loops, 1.0f, cellWidth, false, false);
                    all.push_back(ResultFrame{n, nb, loops, boxDiv, std::move(res)});
                }
            }
        }
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << std::endl;
        return 1;
    }
    std::ofstream file(out.empty() ? default_filename(gensurface) : out);
    file << "NbParticles,NbInteractions,NbLoops,boxDiv,nbCells,partspercell,interactionsperparticle,timeinit,"
            "timecompute,timetotal\n";
    for (const auto& f : all) {
        const long long cells = (long long)f.boxDiv * f.boxDiv * f.boxDiv;
        for (const auto& r : f.results) {
            file << f.nbParticles << "," << f.nbInteractions << "," << f.nbLoops << "," << f.boxDiv << "," << cells
                 << "," << double(f.nbParticles) / cells << "," << double(f.nbInteractions) / f.nbParticles << ","
                 << r.timeInit << "," << r.timeCompute << "," << r.timeTotal << "\n";
        }
    }
    return 0;
}
