// Test driver of the LinearHSC shim: builds the plugin from key=value config
// arguments and, given a system file, runs one do_solve on the GPU.
//   shim_driver <workspace> <system.bin|-> [key=value ...]   (contacts/PT|EE|PE|PP|PH=n: filter sizes)
// system.bin: int64 nnzb, int32 nblock, qo, qm, fo, fn, then rows (int32),
// cols (int32), values (9 doubles per triplet, column-major), b (doubles).
// Writes x to <workspace>/x.bin.  Exit codes: 0 ok, 2 SimSystemException,
// 3 UIPC_ASSERT, 4 I/O.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "linear_hsc_shim.cpp"

using namespace uipc;
using namespace uipc::backend::cuda;

int main(int argc, char** argv) {
    if (argc < 3) return 4;
    Engine eng;
    eng.workspace = argv[1];
    // contacts/PT, /EE, /PE, /PP give the scene a simplex filter, contacts/PH a half-plane filter
    SimplexTrajectoryFilter simplex;
    VertexHalfPlaneTrajectoryFilter half_plane;
    for (int i = 3; i < argc; ++i) {
        std::string kv = argv[i];
        auto eq = kv.find('=');
        std::string k = kv.substr(0, eq), v = kv.substr(eq + 1);
        if (k == "linear_system/solver") eng.w.sc.cfg.strs[k] = v;
        else if (k.rfind("contacts/", 0) == 0) {
            const SizeT n = (SizeT)std::stoll(v);
            if (k == "contacts/PH") { half_plane.ph = n; eng.contacts.half_plane = &half_plane; continue; }
            if (k == "contacts/PT") simplex.pt = n;
            else if (k == "contacts/EE") simplex.ee = n;
            else if (k == "contacts/PE") simplex.pe = n;
            else if (k == "contacts/PP") simplex.pp = n;
            eng.contacts.simplex = &simplex;
        } else eng.w.sc.cfg.nums[k] = std::stod(v);
    }
    auto plugin = make_LinearHSC(eng);
    try {
        plugin->build();
    } catch (const SimSystemException& e) {
        std::cout << "SimSystemException: " << e.what() << "\n";
        return 2;
    } catch (const AssertionError& e) {
        std::cout << "UIPC_ASSERT: " << e.what() << "\n";
        return 3;
    }
    if (std::strcmp(argv[2], "-") == 0) return 0;
    std::ifstream in(argv[2], std::ios::binary);
    if (!in) return 4;
    int64_t nnzb;
    int32_t hdr[5];
    in.read((char*)&nnzb, 8);
    in.read((char*)hdr, sizeof hdr);
    const int nblock = hdr[0];
    eng.abd = {hdr[1], hdr[2]};
    eng.fem = {hdr[3], hdr[4]};
    std::vector<int> rows(nnzb), cols(nnzb);
    std::vector<double> vals(9 * nnzb), b(3 * (size_t)nblock);
    in.read((char*)rows.data(), 4 * nnzb);
    in.read((char*)cols.data(), 4 * nnzb);
    in.read((char*)vals.data(), 72 * nnzb);
    in.read((char*)b.data(), 8 * b.size());
    if (!in) return 4;
    int *dr, *dc;
    double *dv, *db, *dx;
    cudaMalloc(&dr, 4 * nnzb);
    cudaMalloc(&dc, 4 * nnzb);
    cudaMalloc(&dv, 72 * nnzb);
    cudaMalloc(&db, 8 * b.size());
    cudaMalloc(&dx, 8 * b.size());
    cudaMemcpy(dr, rows.data(), 4 * nnzb, cudaMemcpyHostToDevice);
    cudaMemcpy(dc, cols.data(), 4 * nnzb, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, vals.data(), 72 * nnzb, cudaMemcpyHostToDevice);
    cudaMemcpy(db, b.data(), 8 * b.size(), cudaMemcpyHostToDevice);
    GlobalLinearSystem::SolvingInfo info;
    info.m_x = {dx, b.size()};
    info.m_b = {db, b.size()};
    info.m_A = {dr, dc, dv, (SizeT)nnzb, (SizeT)nblock};
    int code = 0;
    try {
        plugin->solve(info);
    } catch (const AssertionError& e) {
        std::cout << "UIPC_ASSERT: " << e.what() << "\n";
        code = 3;
    }
    std::vector<double> x(b.size());
    cudaMemcpy(x.data(), dx, 8 * x.size(), cudaMemcpyDeviceToHost);
    std::ofstream out(eng.workspace + "/x.bin", std::ios::binary);
    out.write((const char*)x.data(), 8 * x.size());
    std::cout << "iterations " << info.m_iters << "\n";
    cudaFree(dr); cudaFree(dc); cudaFree(dv); cudaFree(db); cudaFree(dx);
    return code;
}
