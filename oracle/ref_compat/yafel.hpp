// yafel.hpp -- stand-in for the reference's convenience header
// (include/yafel.hpp), found first on the oracle's include path.  It includes
// only the reference headers that apps/supg_learning/supg_advection.hpp needs
// (the full header also pulls in ViennaCL solvers and output writers, which
// need libraries that are not installed).  TEST INFRASTRUCTURE ONLY.
#ifndef _YAFEL_HPP
#define _YAFEL_HPP
#include "yafel_globals.hpp"
#include "lin_alg/tensor/tensors.hpp"
#include "assembly/CGAssembly.hpp"
#include "boundary_conditions/DirichletBC.hpp"
#include "fe_system/FESystem.hpp"
#include "quadrature/QuadratureRule.hpp"
#include "utils/DoFManager.hpp"
#include "PDE/PDEBase.hpp"
#include "mesh/Mesh.hpp"
#include "element/Element.hpp"
#include "element/ElementFactory.hpp"
#include "element/ElementType.hpp"
#include "element/ShapeFunctionUtils.hpp"
#endif
