// Declarations that the reference's dc_backend.cpp takes from its contouring.h, reduced to
// what compiles without Eigen (see Eigen/Core beside this file). TEST INFRASTRUCTURE ONLY.
#pragma once
#include <functional>
#include <unordered_map>   // the real header chain brings it in; dc_backend.cpp relies on that
#include <vector>
#include <Eigen/Core>

enum class ContouringMethod { MarchingCubes, DualContouring, Ours };

struct ContouringOptions {
    ContouringMethod method = ContouringMethod::DualContouring;
    bool verbose = false;
};

void contouring(const Eigen::VectorXd& S, const Eigen::MatrixXd& GV, int resX, int resY, int resZ, double isoValue,
                Eigen::MatrixXd& V, Eigen::MatrixXi& F, const ContouringOptions& options);

std::vector<class Cell>* getGeneratedCells();
