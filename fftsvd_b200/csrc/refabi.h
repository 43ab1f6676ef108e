// Memory layout of the reference FFTSVD host structures, as built by the
// reference with its default configuration (REAL_IS_DOUBLE, SREAL_IS_FLOAT,
// LOCAL 1, no ADAPTIVE / SERIALIZE / SCATTER / POLYNOMIAL / ENABLE_GALERKIN;
// FFTSVD.h:23-103) on an LP64 platform.  The drop-in entry points read a
// caller's reference-built SurfaceOperator through these mirrors; field order
// and types must match the reference headers exactly:
//   Vector3D.h:3-7  Panel.h:3-25  FlatPanel.h:3-27  Charge.h:3-8  Tree.h:3-38
//   Cube.h:3-54  SurfaceOperator.h:5-23  Preconditioner.h:3-17 (leading fields)
//   FFTSVDpbeAPI.h:23-42 (PDBentry)
#pragma once

#include <cstdint>

namespace fftsvd {
namespace ref {

typedef double real;
typedef float sreal;

struct Vec3 {
   real x, y, z;
};

struct Panel {
   Vec3* centroid;
   Vec3* normal;
   real area;
   real maxedgelength;
   unsigned int numdirectquadpoints;
   Vec3** directquadpoints;
   Vec3** directquadnormals;
   real* directquadweights;
   int type;  // PanelType: FLAT_PANEL == 0
   void* realpanel;
};

struct FlatPanel {  // leading field only
   Vec3* vertex[3];
};

struct Charge {
   unsigned int numcharges;
   unsigned int globalindexstart;
   Vec3** points;
   real* charges;
};

struct Cube;

struct Tree {
   Panel** panels;
   unsigned int numpanels;
   Vec3** points;
   Vec3** normals;
   unsigned int numpoints;
   unsigned int maxpanelsperfinestcube;
   unsigned int partitioningdepth;
   int kerneltype;
   void* parameters;
   unsigned int gridpoints;
   unsigned int* gridpointsperlevel;
   real (*quadraturepoints)[4];
   unsigned int numquadraturepoints;
   real** pinv_Q2Sgridpoints;
   real epsilon;
   int layertype;
   float***** Tprecomputed;  // [level][x+3][y+3][z+3] -> padded grid, (re, im) float pairs
   Cube* root;
   real minimumcubesize;
};

struct Cube {
   unsigned int level;
   unsigned int indices[3];
   Vec3* bounds[2];
   Vec3* center;
   Cube* parent;
   unsigned int leaf;
   unsigned int* panelindices;
   unsigned int numpanelindices;
   unsigned int* pointindices;
   unsigned int numpointindices;
   Cube** localcubes;
   unsigned int numlocalcubes;
   Cube** interactingcubes;
   unsigned int numinteractingcubes;
   Cube* children[2][2][2];
   unsigned int drows, dcolumns;
   unsigned int rowrank, columnrank;
   sreal** VTsrc;
   sreal** Udest;
   sreal** D_single;
   sreal** D_double;
   void* FFT_PV_VT_q;
   void* sum_T_FFT_PV_VT_q;
   void* FFT_UTIT_UT_q;
   void* sum_T_FFT_UTIT_UT_q;
   sreal** UTI;
   sreal** PV_single;
   sreal** PV_double;
   sreal** P_single;
   sreal** P_double;
   sreal** I_;
   sreal** I_double;
   Tree* tree;
};

struct SurfaceOperator {
   int kernel;
   real epsilon;
   real kappa;
   unsigned int mynumpanels;
   unsigned int startphi;
   unsigned int startdphi;
   Tree* tree;
   Tree* M3;
   unsigned int numchildren;
   SurfaceOperator** children;
   real* resultInternal;
   real* resultExternal;
   SurfaceOperator* parent;
   Charge* charges;
};

struct PreconditionerElement {
   unsigned int row;
   real value;
};

struct Preconditioner {  // leading fields only; SuperLU factors follow
   unsigned int rows, columns, nnz;
   PreconditionerElement** P;
   unsigned int* numelements;
};

// One atom of the reference PBE API: read and written by collectPotentials.
struct PDBentry {
   char record[7];
   unsigned int atomnumber;
   char atomname[5];
   char alternatelocation;
   char residuename[4];
   char chain;
   unsigned int residuenumber;
   char residueinsertion;
   real x, y, z;
   real occupancy;
   real temperature;
   unsigned int footnotenumber;
   real radius;
   real charge;
   real potential;
};

}  // namespace ref
}  // namespace fftsvd
