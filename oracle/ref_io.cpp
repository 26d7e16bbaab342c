/*
 * ORACLE TEST INFRASTRUCTURE — not part of the product.
 *
 * The reference's grid output writer on an arbitrary state: toNaturalData
 * (conversions.cpp:37-57) and outputGridData -> outputGridDataBinary
 * (file_access.cpp:1530-1677, 1193-1325), as main.cpp:301-303 calls them at
 * an output step, writing to a temporary file whose bytes are handed back.
 * The checker of the device grid-dump pack (mhd_grid_pack).  Linked with the
 * reference's whole program except main.cpp, compiled unmodified with the
 * project-written Boost stand-in headers (see oracle/Makefile); nothing of
 * the reference is copied here.
 */
#include "mhd2d.hpp"

#include <cstdio>
#include <vector>

namespace {

/* Pointer tables that view one contiguous [k][i][j] block as t_matrices. */
struct Planes {
   std::vector<double*> rows;
   std::vector<double**> planes;
   Planes( double* base, int n, int sx, int sy ) : rows( size_t(n)*sx ), planes( n ) {
      for( int k = 0; k < n; k++ ){
         planes[k] = &rows[size_t(k)*sx];
         for( int i = 0; i < sx; i++ )
            rows[size_t(k)*sx+i] = base + (size_t(k)*sx+i)*sy;
      }
   }
};

BoundaryCondition bcOf( int v ){
   switch( v ){
   case 1: return BoundaryCondition::Periodic;
   case 2: return BoundaryCondition::Dirichlet;
   case 3: return BoundaryCondition::Neumann;
   case 4: return BoundaryCondition::Open;
   default: return BoundaryCondition::Undefined;
   }
}

} // namespace

/* The reference program defines this in main.cpp (main.cpp:365-396), which is
   not linked here; the writer only calls it on a file it cannot open. */
void criticalError( ReturnStatus error, const std::string message ){
   std::fprintf( stderr, "Critical error (%d): %s\n", int( error ), message.c_str() );
   std::abort();
}

extern "C" {

/* The bytes outputGridData writes for state U ([8][nx+4][ny+4], ghosts
   included; the writer overwrites the B ghosts of periodic and open sides in
   place, as it does in the reference's main loop).  bc order: left, right,
   bottom, top.  Returns the byte count, or -1 if out_bytes is too small. */
long long ref_grid_records( int nx, int ny, double dx, double dy, double gamma, double start_x,
                            double start_y, const int* bc, double* U, int natural,
                            int conservation, int binary_double, void* out, long long out_bytes )
{
   t_params params{};
   params.nx = nx; params.ny = ny; params.dx = dx; params.dy = dy; params.gamma = gamma;
   params.start_x = start_x; params.start_y = start_y;
   params.boundary[params.b_left]   = bcOf( bc[0] );
   params.boundary[params.b_right]  = bcOf( bc[1] );
   params.boundary[params.b_bottom] = bcOf( bc[2] );
   params.boundary[params.b_top]    = bcOf( bc[3] );
   const int NXt = nx+4, NYt = ny+4;
   std::vector<double> ubuf( size_t(VEL_DIM)*NXt*NYt ), pbuf( size_t(NXt)*NYt );
   Planes vU( U, PRB_DIM, NXt, NYt ), vu( ubuf.data(), VEL_DIM, NXt, NYt ),
          vp( pbuf.data(), 1, NXt, NYt );
   t_data data{};
   data.U = vU.planes.data();
   data.u = vu.planes.data();
   data.p = vp.planes[0];
   data.t_current = 0.0;
   toNaturalData( params, data );

   t_output output{};
   output.binary = true;
   output.binary_double = binary_double != 0;
   output.single_file = true;
   output.natural = natural != 0;
   output.conservation = conservation != 0;
   output.file = std::tmpfile();
   if( !output.file ) return -1;
   outputGridData( output, params, data, 0, 0 );
   std::fflush( output.file );
   const long n = std::ftell( output.file );
   long long got = -1;
   if( n >= 0 && n <= out_bytes ){
      std::rewind( output.file );
      got = (long long)std::fread( out, 1, size_t(n), output.file );
   }
   std::fclose( output.file );
   return got;
}

} // extern "C"
