// A C++ program written against the reference-shaped adapters
// (include/dfm_b200_lsol.hpp) and the C ABI only: 2-D Poisson on the unit
// square (n x n grid of P1 triangles, u = 0 on the boundary), assembled on the
// device, ILU(0)-PCG and ILU(0)-PBiCGSTAB.  Prints one JSON object with the
// iteration counts, convergence ratios and the PCG solution.
//
//   g++ -std=c++17 -Iinclude tests/cpp/lsol_demo.cpp -Ldelfem_b200/_lib -ldfm_b200 -o lsol_demo
//   ./lsol_demo 16 > out.json
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "dfm_b200_lsol.hpp"

int main(int argc, char** argv) {
  const int n = argc > 1 ? std::atoi(argv[1]) : 16;
  const int m = n + 1;
  std::vector<double> coord;
  std::vector<int> elem, fixed;
  for (int j = 0; j < m; j++)
    for (int i = 0; i < m; i++) {
      coord.push_back((double)i / n);
      coord.push_back((double)j / n);
      fixed.push_back(i == 0 || j == 0 || i == n || j == n);
    }
  for (int j = 0; j < n; j++)  // the same triangles as delfem_b200.meshes.unit_square_tri
    for (int i = 0; i < n; i++) {
      const int p = i + j * m;
      const int t[6] = {p, p + 1, p + m + 1, p, p + m + 1, p + m};
      elem.insert(elem.end(), t, t + 6);
    }
  try {
    dfm_lsol::Context ctx(0);
    dfm_mesh mesh = nullptr;
    dfm_lsol::check(dfm_mesh_create(ctx.get(), 2, m * m, coord.data(), 3, 2 * n * n, elem.data(), 0, nullptr, &mesh),
                    "dfm_mesh_create");
    size_t ncrs = 0;
    std::vector<unsigned> rp(m * m + 1);
    dfm_lsol::check(dfm_mesh_pattern(mesh, rp.data(), nullptr, &ncrs), "pattern size");
    std::vector<unsigned> ci(ncrs);
    dfm_lsol::check(dfm_mesh_pattern(mesh, rp.data(), ci.data(), &ncrs), "pattern");
    dfm_lsol::CMatDia_BlkCrs A(ctx, m * m, 1, rp.data(), ci.data());
    dfm_lsol::DeviceVector f(ctx, A.VectorSize()), r(ctx, A.VectorSize()), x(ctx, A.VectorSize());
    void* flags = nullptr;
    dfm_lsol::check(dfm_buf_alloc(ctx.get(), fixed.size() * sizeof(int), &flags), "alloc");
    dfm_lsol::check(dfm_buf_copy(ctx.get(), flags, fixed.data(), fixed.size() * sizeof(int), DFM_H2D), "copy");
    dfm_lsol::check(dfm_assemble_poisson2d(mesh, A.get(), 1.0, 1.0, nullptr, nullptr, nullptr, f.data()), "assemble");
    dfm_lsol::check(dfm_apply_dirichlet(A.get(), static_cast<const int*>(flags), f.data()), "dirichlet");
    dfm_lsol::CPreconditioner_ILU M(A);
    if (!M.SetValue(A)) return 2;
    double conv = 1e-10;
    unsigned it = 1000;
    r.copy_from(f);
    const bool ok = dfm_lsol::Solve_PCG(conv, it, A, M, r, x);
    std::vector<double> xh(A.VectorSize());
    x.download(xh.data());
    double conv2 = 1e-10;
    unsigned it2 = 1000;
    dfm_lsol::DeviceVector x2(ctx, A.VectorSize());
    r.copy_from(f);
    const bool ok2 = dfm_lsol::Solve_PBiCGSTAB(conv2, it2, A, M, r, x2);
    // ILU(1): CPreconditioner_ILU::SetFillInLevel before SetLinearSystem
    dfm_lsol::CPreconditioner_ILU M1;
    M1.SetFillInLevel(1);
    M1.SetLinearSystem(A);
    if (!M1.SetValue(A)) return 2;
    double conv3 = 1e-10;
    unsigned it3 = 1000;
    dfm_lsol::DeviceVector x3(ctx, A.VectorSize());
    r.copy_from(f);
    const bool ok3 = dfm_lsol::Solve_PCG(conv3, it3, A, M1, r, x3);
    std::vector<double> xh3(A.VectorSize());
    x3.download(xh3.data());
    // ILU(1) with unlimited fill through every 7th block row of the middle
    // third: CPreconditioner_ILU::SetFillBlk
    dfm_lsol::CPreconditioner_ILU M2;
    M2.SetFillInLevel(1);
    std::vector<unsigned int> blk;
    for (unsigned i = A.NBlkMatCol() / 3; i < 2 * A.NBlkMatCol() / 3; i += 7) blk.push_back(i);
    M2.SetFillBlk(blk);
    M2.SetLinearSystem(A);
    if (!M2.SetValue(A)) return 2;
    double conv4 = 1e-10;
    unsigned it4 = 1000;
    dfm_lsol::DeviceVector x4(ctx, A.VectorSize());
    r.copy_from(f);
    const bool ok4 = dfm_lsol::Solve_PCG(conv4, it4, A, M2, r, x4);
    std::vector<double> xh4(A.VectorSize());
    x4.download(xh4.data());
    std::printf("{\"pcg_ok\": %s, \"pcg_iters\": %u, \"pcg_conv\": %.17g, \"bicg_ok\": %s, \"bicg_iters\": %u, "
                "\"bicg_conv\": %.17g, \"ilu1_ok\": %s, \"ilu1_iters\": %u, \"fillblk_ok\": %s, "
                "\"fillblk_iters\": %u, \"x\": [",
                ok ? "true" : "false", it, conv, ok2 ? "true" : "false", it2, conv2, ok3 ? "true" : "false", it3,
                ok4 ? "true" : "false", it4);
    for (size_t k = 0; k < xh.size(); k++) std::printf("%s%.17g", k ? ", " : "", xh[k]);
    std::printf("], \"x_ilu1\": [");
    for (size_t k = 0; k < xh3.size(); k++) std::printf("%s%.17g", k ? ", " : "", xh3[k]);
    std::printf("], \"x_fillblk\": [");
    for (size_t k = 0; k < xh4.size(); k++) std::printf("%s%.17g", k ? ", " : "", xh4[k]);
    std::printf("]");
    // optional: a complex matrix in the reference's text format (argv[2]) and
    // its right-hand side (argv[3], one "re im" pair per row), solved by PCOCG
    if (argc > 3) {
      dfm_lsol::CMatDia_BlkCrs Z = dfm_lsol::CMatDia_BlkCrs::FromTextFile(ctx, argv[2]);
      std::vector<double> bh(Z.VectorSize());
      FILE* fb = std::fopen(argv[3], "r");
      if (!fb) return 3;
      for (double& v : bh)
        if (std::fscanf(fb, "%lf", &v) != 1) { std::fclose(fb); return 3; }
      std::fclose(fb);
      dfm_lsol::CPreconditioner_ILU MZ(Z);
      if (!MZ.SetValue(Z)) return 2;
      dfm_lsol::DeviceVector rz(ctx, Z.VectorSize()), xz(ctx, Z.VectorSize());
      rz.upload(bh.data());
      double convz = 1e-10;
      unsigned itz = 3000;
      const bool okz = dfm_lsol::Solve_PCOCG(convz, itz, Z, MZ, rz, xz);
      std::vector<double> xzh(Z.VectorSize());
      xz.download(xzh.data());
      std::printf(", \"pcocg_ok\": %s, \"pcocg_iters\": %u, \"x_file\": [", okz ? "true" : "false", itz);
      for (size_t k = 0; k < xzh.size(); k++) std::printf("%s%.17g", k ? ", " : "", xzh[k]);
      std::printf("]");
    }
    std::printf("}\n");
    dfm_buf_free(ctx.get(), flags);
    dfm_mesh_destroy(mesh);
  } catch (const dfm_lsol::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
