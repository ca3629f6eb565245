// Drives the reference-style C++ interface (include/mpm_simulator.hpp) the way
// the reference's main() does (src/main.cpp:161-221): build objects, step,
// read positions, write a .bgeo frame.  Prints one JSON line.
//   shim_demo <shape-or-obj-path> <substeps> <bgeo-out>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "mpm_simulator.hpp"

int main(int argc, char** argv) {
    const std::string shape = argc > 1 ? argv[1] : "builtin:cube";
    const int steps = argc > 2 ? std::atoi(argv[2]) : 10;
    const std::string out = argc > 3 ? argv[3] : "Frame000001.bgeo";
    try {
        std::vector<ObjInitInfo> infos;
        ObjInitInfo a;
        a.objPath = shape;
        a.initVel = {0.0, -1.0, 0.0};
        a.initScale = mpm_shim::vec3(0.2f, 0.2f, 0.2f);
        a.initTranslation = mpm_shim::vec3(0.5f, 0.5f, 0.5f);
        a.initRotationAxis = mpm_shim::vec3(0.f, 1.f, 0.f);
        a.initRotationDegree = 30.f;
        a.mMaterial = Material(5e4, 0.3, 1000.0, JELLO);
        infos.push_back(a);
        ObjInitInfo b = a;
        b.objPath = "builtin:sphere";
        b.initTranslation = mpm_shim::vec3(0.5f, 0.25f, 0.5f);
        b.initVel = {0.0, 0.0, 0.0};
        b.mMaterial = Material(5e3, 0.3, 1000.0, WATER);
        infos.push_back(b);
        MPMSimulator sim(1.0 / 64, 1e-4, 64, 64, 64, 4, infos);
        const int n = sim.totalParticlesNum();
        for (int i = 0; i < steps; ++i) sim.step();
        std::vector<float> pos;
        sim.getGLParticlesPos(pos);
        OutputBego(out, pos);
        double mean[3] = {0, 0, 0};
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) mean[k] += pos[3 * i + k] / n;
        std::printf("{\"particles\": %d, \"frame\": %d, \"time\": %.6f, \"mean\": [%.7f, %.7f, %.7f]}\n", n,
                    sim.current_frame, sim.current_time, mean[0], mean[1], mean[2]);
    } catch (const std::exception& e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 1;
    }
    return 0;
}
