// Compatibility header: the reference's umbrella include (LoAdSG's
// library/source/sparseEXPDE.h) for programs written against LoAdSG, on top of
// the C++ drop-in loadsg.hpp and liblsg.so.  With
//     -I <this repository>/include/loadsg/compat -DDimensionSparseGrid=<d>
// a LoAdSG main that uses the prewavelet path compiles unchanged: its
// `#include "source/sparseEXPDE.h"` finds this file.
//
// The reference fixes the dimension at compile time (abbrevi.h:11,
// `#define DimensionSparseGrid 3`); the names below are the drop-in's
// templates at that dimension:
//   IndexDimension                 indices/index.h:489+ (center point, coordinate(d))
//   AdaptiveSparseGrid             sgrid/sparseGrid.h:86-387
//   MultiLevelAdaptiveSparseGrid   sgrid/multilevelSparseGrid.h:13-143
//   VectorSparseG                  extemp/vector.h:247-441 (+, -, scalar * of vectors)
//   MatrixVectorHomogen            MatrixVectorMultiplication/MatrixVectorHomogen.h:32-652
//   Poisson, HelmHoltz             stencils/Stencil.h:1605-1793, 873-919
//   CG::solveHomogen               applications/cg_method.h:27-33
//   calcPrewByNodal, calcNodalByPrew   BasisTransformations/BasisTransformations.h:117,123
//   L2, H1, L_infty                applications/H1_Norm.h, applications/norms.h
// Everything runs on the GPU through the C-ABI; there is no CPU fallback.
#pragma once

#ifndef DimensionSparseGrid
#define DimensionSparseGrid 3
#endif

#include <cmath>
#include <iostream>
#include <string>

#include "../../loadsg.hpp"

// the reference's headers bring std into the global namespace
// (sgrid/simpleMultiHash.h:7); its mains rely on it
using namespace std;

// A point of the grid by its 1D indices (index.h: root 2, sons 2i and 2i+1,
// boundary 0 and 1); the default is the center point.
class IndexDimension {
public:
    IndexDimension() { idx_.fill(2); }
    explicit IndexDimension(const std::array<int32_t, DimensionSparseGrid>& i) : idx_(i) {}
    int32_t getIndex(int d) const { return idx_[d]; }
    void replace(int d, int32_t i) { idx_[d] = i; }
    // index.h:718-730: i = 0 -> 0, i = 1 -> 1, else (2 (i - 2^t) + 1) / 2^t at depth t
    double coordinate(int d) const {
        int32_t i = idx_[d];
        if (i < 2) return (double)i;
        int t = 31 - __builtin_clz((unsigned)i);
        return (2.0 * (i - (1 << t)) + 1.0) / (double)(1 << t);
    }
    const std::array<int32_t, DimensionSparseGrid>& indices() const { return idx_; }

private:
    std::array<int32_t, DimensionSparseGrid> idx_;
};

class AdaptiveSparseGrid : public lsg::AdaptiveSparseGrid<DimensionSparseGrid> {
    using Base = lsg::AdaptiveSparseGrid<DimensionSparseGrid>;

public:
    using Base::AddRecursiveSonsOfPoint;
    void AddRecursiveSonsOfPoint(const IndexDimension& center, int level) {
        Base::AddRecursiveSonsOfPoint(center.indices(), level);
    }
    bool AddPoint(const IndexDimension& I) { return Base::AddPoint(I.indices()); }
    IndexDimension getIndexOfTable(unsigned long k) const { return IndexDimension(Base::getIndexOfTable((int64_t)k)); }
    unsigned long getMaximalOccupiedSecondTable() const { return (unsigned long)Base::getMaximalOccupiedSecondTable(); }
};

using MultiLevelAdaptiveSparseGrid = lsg::MultiLevelAdaptiveSparseGrid<DimensionSparseGrid>;
using VectorSparseG = lsg::VectorSparseG<DimensionSparseGrid>;
using MatrixVectorHomogen = lsg::MatrixVectorHomogen<DimensionSparseGrid>;
using Poisson = lsg::Poisson;
using HelmHoltz = lsg::HelmHoltz;
using CG = lsg::CG;
using L2 = lsg::L2<DimensionSparseGrid>;
using H1 = lsg::H1<DimensionSparseGrid>;

inline void calcPrewByNodal(VectorSparseG& prew, const VectorSparseG& u) { lsg::calcPrewByNodal<DimensionSparseGrid>(prew, u); }
inline void calcNodalByPrew(const VectorSparseG& prew, VectorSparseG& u) { lsg::calcNodalByPrew<DimensionSparseGrid>(prew, u); }
inline double L_infty(const VectorSparseG& v) { return lsg::L_infty<DimensionSparseGrid>(v); }
