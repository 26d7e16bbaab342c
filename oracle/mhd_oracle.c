/*
 * ORACLE — TEST INFRASTRUCTURE ONLY (see mhd_oracle.h).  CPU restatement of
 * the reference hot path, used as the checker by tests/, the smoke check and
 * bench.py's cpu_baseline leg.  Never linked into the product.
 *
 * Arithmetic note.  Every floating-point expression keeps the association
 * order of the reference formula it restates (C evaluates a*b*c as (a*b)*c,
 * a-b-c as (a-b)-c), and the file is compiled with -ffp-contract=off, so the
 * oracle reproduces the reference bit for bit (x86-64 SSE2 doubles, IEEE
 * division and square root on both sides).
 */
#include "mhd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NF 8
#define SMALL 1e-20 /* EPS of mhd2d.hpp:76 */

struct orc_ctx {
   int scheme, time_method;
   int nx, ny, NX, NY;
   double dx, dy, gamma;
   int bc[4];                 /* left, right, bottom, top */
   double dt_min, dt_max, cfl;
   int dirichlet_needed;      /* some side is Dirichlet and no snapshot yet */
   double *dl, *dr, *db, *dt; /* Dirichlet snapshots [8][NY] / [8][NX] */
   double *F, *G;             /* physical fluxes */
   double *VF, *VG;           /* undivided differences (ENO-Roe) */
   double *FN, *GN;           /* numerical fluxes at interfaces */
   double *cx, *cy, *LUx, *LUy;
   double *aF, *aG;           /* ENO-LF dissipation [8][NY] / [8][NX] */
   int alpha_fixed;           /* aF / aG set by orc_set_lf_alpha: integrate keeps them */
   double *U1, *U2, *UL;      /* time-stepper stages */
   double *phi;               /* SOR potential, persists across solves */
   long long retries;         /* RK3 stage restarts taken so far */
   int cfd_i, cfd_j;          /* central FD: cell of the reported density / pressure error */
};

enum { L = 0, R = 1, B = 2, T = 3 };
enum { PER = 1, DIR = 2, NEU = 3, OPN = 4 };

#define AT(a,k,i,j) (a)[((size_t)(k)*c->NX + (size_t)(i))*c->NY + (size_t)(j)]
#define PHI(i,j)    c->phi[(size_t)(i)*c->NY + (size_t)(j)]

static double* zalloc( size_t n ){ return (double*)calloc( n, sizeof(double) ); }

orc_ctx* orc_create( int scheme, int time_method, int nx, int ny, double dx, double dy,
                     double gamma, const int* bc, double dt_min, double dt_max, double cfl )
{
   orc_ctx* c = (orc_ctx*)calloc( 1, sizeof *c );
   size_t tot;
   c->scheme = scheme; c->time_method = time_method;
   c->nx = nx; c->ny = ny; c->NX = nx+4; c->NY = ny+4;
   c->dx = dx; c->dy = dy; c->gamma = gamma;
   memcpy( c->bc, bc, sizeof c->bc );
   c->dt_min = dt_min; c->dt_max = dt_max; c->cfl = cfl;
   c->dirichlet_needed = bc[0] == DIR || bc[1] == DIR || bc[2] == DIR || bc[3] == DIR;
   tot = (size_t)NF*c->NX*c->NY;
   c->dl = zalloc( (size_t)NF*c->NY ); c->dr = zalloc( (size_t)NF*c->NY );
   c->db = zalloc( (size_t)NF*c->NX ); c->dt = zalloc( (size_t)NF*c->NX );
   c->F = zalloc( tot ); c->G = zalloc( tot ); c->VF = zalloc( tot ); c->VG = zalloc( tot );
   c->FN = zalloc( tot ); c->GN = zalloc( tot );
   c->cx = zalloc( tot ); c->cy = zalloc( tot ); c->LUx = zalloc( tot ); c->LUy = zalloc( tot );
   c->aF = zalloc( (size_t)NF*c->NY ); c->aG = zalloc( (size_t)NF*c->NX );
   c->U1 = zalloc( tot ); c->U2 = zalloc( tot ); c->UL = zalloc( tot );
   c->phi = zalloc( (size_t)c->NX*c->NY );
   return c;
}

void orc_destroy( orc_ctx* c )
{
   double* bufs[] = { c->dl, c->dr, c->db, c->dt, c->F, c->G, c->VF, c->VG, c->FN, c->GN,
                      c->cx, c->cy, c->LUx, c->LUy, c->aF, c->aG, c->U1, c->U2, c->UL, c->phi };
   size_t n;
   if( !c ) return;
   for( n = 0; n < sizeof bufs / sizeof bufs[0]; n++ ) free( bufs[n] );
   free( c );
}

/* spatialintegrationmethod.cpp:39-59 — edge rows/columns of the interior. */
void orc_init_dirichlet( orc_ctx* c, const double* U )
{
   int k, i, j;
   for( k = 0; k < NF; k++ ){
      for( i = 2; i < c->nx+2; i++ ){
         c->db[(size_t)k*c->NX+i] = AT(U,k,i,2);
         c->dt[(size_t)k*c->NX+i] = AT(U,k,i,c->ny+1);
      }
      for( j = 2; j < c->ny+2; j++ ){
         c->dl[(size_t)k*c->NY+j] = AT(U,k,2,j);
         c->dr[(size_t)k*c->NY+j] = AT(U,k,c->nx+1,j);
      }
   }
   c->dirichlet_needed = 0;
}

/* spatialintegrationmethod.cpp:85-300.  Sides in the order left, right,
   bottom, top; ghost layer g = 1, 2 counts outward from the edge.  Neumann
   adds the div B = 0 extrapolation of the normal field into the ghosts. */
int orc_apply_bc( orc_ctx* c, double* U, int* is_error )
{
   const int nx = c->nx, ny = c->ny, f0 = 2, lx = nx+2, ly = ny+2;
   int k, g, i, j;
   *is_error = 0;
   if( c->dirichlet_needed ){ *is_error = 1; return ORC_ERR_WRONG_PARAMETER; }
   for( k = 0; k < 4; k++ ) if( c->bc[k] < PER || c->bc[k] > OPN ){ *is_error = 1; return ORC_ERR_WRONG_PARAMETER; }

   /* left */
   for( k = 0; k < NF; k++ ) for( g = 1; g <= 2; g++ ) for( j = f0; j < ly; j++ ){
      double v;
      switch( c->bc[L] ){
      case PER: v = AT(U,k,lx-g,j); break;
      case DIR: v = c->dl[(size_t)k*c->NY+j]; break;
      default:  v = AT(U,k,f0+g,j); break;   /* Neumann, open: mirror */
      }
      AT(U,k,f0-g,j) = v;
   }
   if( c->bc[L] == NEU ){
      const double rxy = c->dx/c->dy;
      for( i = f0; i > 0; i-- ) for( j = f0+1; j < ly-1; j++ )
         AT(U,4,i-1,j) = AT(U,4,i+1,j) - rxy*( AT(U,5,i,j-1) - AT(U,5,i,j+1) );
   }
   /* right */
   for( k = 0; k < NF; k++ ) for( g = 1; g <= 2; g++ ) for( j = f0; j < ly; j++ ){
      double v;
      switch( c->bc[R] ){
      case PER: v = AT(U,k,f0-1+g,j); break;
      case DIR: v = c->dr[(size_t)k*c->NY+j]; break;
      default:  v = AT(U,k,lx-1-g,j); break;
      }
      AT(U,k,lx-1+g,j) = v;
   }
   if( c->bc[R] == NEU ){
      const double rxy = c->dx/c->dy;
      for( i = lx-1; i < c->NX-1; i++ ) for( j = f0+1; j < ly-1; j++ )
         AT(U,4,i+1,j) = AT(U,4,i-1,j) - rxy*( AT(U,5,i,j+1) - AT(U,5,i,j-1) );
   }
   /* bottom */
   for( k = 0; k < NF; k++ ) for( i = f0; i < lx; i++ ) for( g = 1; g <= 2; g++ ){
      double v;
      switch( c->bc[B] ){
      case PER: v = AT(U,k,i,ly-g); break;
      case DIR: v = c->db[(size_t)k*c->NX+i]; break;
      default:  v = AT(U,k,i,f0+g); break;
      }
      AT(U,k,i,f0-g) = v;
   }
   if( c->bc[B] == NEU ){
      const double ryx = c->dy/c->dx;
      for( i = f0+1; i < lx-1; i++ ) for( j = f0; j > 0; j-- )
         AT(U,5,i,j-1) = AT(U,5,i,j+1) - ryx*( AT(U,4,i-1,j) - AT(U,4,i+1,j) );
   }
   /* top */
   for( k = 0; k < NF; k++ ) for( i = f0; i < lx; i++ ) for( g = 1; g <= 2; g++ ){
      double v;
      switch( c->bc[T] ){
      case PER: v = AT(U,k,i,f0-1+g); break;
      case DIR: v = c->dt[(size_t)k*c->NX+i]; break;
      default:  v = AT(U,k,i,ly-1-g); break;
      }
      AT(U,k,i,ly-1+g) = v;
   }
   if( c->bc[T] == NEU ){
      const double ryx = c->dy/c->dx;
      for( i = f0+1; i < lx-1; i++ ) for( j = ly-1; j < c->NY-1; j++ )
         AT(U,5,i,j+1) = AT(U,5,i,j-1) - ryx*( AT(U,4,i+1,j) - AT(U,4,i-1,j) );
   }
   return ORC_OK;
}

/* spatialmethodeno.cpp:89-127 — physical fluxes at every cell. */
static void fluxes( orc_ctx* c, const double* U )
{
   const double gm = c->gamma;
   int i, j;
   for( i = 0; i < c->NX; i++ ) for( j = 0; j < c->NY; j++ ){
      const double r = AT(U,0,i,j), mx = AT(U,1,i,j), my = AT(U,2,i,j), mz = AT(U,3,i,j);
      const double bx = AT(U,4,i,j), by = AT(U,5,i,j), bz = AT(U,6,i,j), e = AT(U,7,i,j);
      const double u = mx/r, v = my/r, w = mz/r;
      const double uu = u*u + v*v + w*w;
      const double ub = u*bx + v*by + w*bz;
      const double bb = bx*bx + by*by + bz*bz;
      const double p = (gm-1.0)*(e - 0.5*r*uu - 0.5*bb);
      const double pt = p + 0.5*bb;
      AT(c->F,0,i,j) = mx;               AT(c->G,0,i,j) = my;
      AT(c->F,1,i,j) = mx*u - bx*bx + pt; AT(c->G,1,i,j) = mx*v - by*bx;
      AT(c->F,2,i,j) = my*u - bx*by;     AT(c->G,2,i,j) = my*v - by*by + pt;
      AT(c->F,3,i,j) = mz*u - bx*bz;     AT(c->G,3,i,j) = mz*v - by*bz;
      AT(c->F,4,i,j) = 0;                AT(c->G,4,i,j) = bx*v - by*u;
      AT(c->F,5,i,j) = by*u - bx*v;      AT(c->G,5,i,j) = 0;
      AT(c->F,6,i,j) = bz*u - bx*w;      AT(c->G,6,i,j) = bz*v - by*w;
      AT(c->F,7,i,j) = (e+pt)*u - bx*ub; AT(c->G,7,i,j) = (e+pt)*v - by*ub;
   }
}

/* spatialmethodeno.cpp:130-206 — cell-centred eigenvalues.
   Returns 1 on non-positive density; *neg_pressure = 1 when p was clamped. */
int orc_eigenvalues_at( double gm, const double* U, double* lam, int* neg_pressure )
{
   const double r = U[0], mx = U[1], u = U[1]/U[0], my = U[2], mz = U[3];
   const double bx = U[4], by = U[5], bz = U[6], e = U[7];
   double mm, bb, p, a2, ca2, ca, c2, ct, cs2, cs, cf2, cf;
   *neg_pressure = 0;
   if( r <= 0.0 ) return 1;
   mm = mx*mx + my*my + mz*mz;
   bb = bx*bx + by*by + bz*bz;
   p = (gm-1.0)*( e - 0.5*mm/r - 0.5*bb );
   if( p < 0.0 ){ p = 0.0; *neg_pressure = 1; }
   a2 = gm*p / r;      if( a2 < 0.0 ) a2 = 0.0;
   ca2 = bx*bx/r;      ca = sqrt( ca2 );
   c2 = 0.5*(bb/r+a2);
   ct = c2*c2-a2*ca2;  if( ct < 0.0 ) ct = 0.0;
   cs2 = c2 - sqrt(ct); if( cs2 < 0.0 ) cs2 = SMALL;
   cs = sqrt( cs2 );
   cf2 = c2 + sqrt(ct); if( cf2 < 0.0 ) cf2 = SMALL;
   cf = sqrt( cf2 );
   lam[0] = u - cf; lam[1] = u - ca; lam[2] = u - cs; lam[3] = u;
   lam[4] = u + cs; lam[5] = u + ca; lam[6] = u + cf; lam[7] = 0;
   return 0;
}

/* spatialmethodeno.cpp:288-571 — eigen-decomposition at the arithmetic-mean
   midpoint of U1 and U2 (x direction).  lv, rv are row-major 8x8 (row =
   characteristic).  Returns 1 on non-positive midpoint density. */
int orc_eigens_f( double gm, const double* U1, const double* U2, double* lam,
                  double* lv, double* rv, int* neg_pressure )
{
   const double r  = 0.5 * ( U1[0] + U2[0] );
   const double u  = 0.5 * ( U1[1]/U1[0] + U2[1]/U2[0] );
   const double v  = 0.5 * ( U1[2]/U1[0] + U2[2]/U2[0] );
   const double w  = 0.5 * ( U1[3]/U1[0] + U2[3]/U2[0] );
   const double bx = 0.5 * ( U1[4] + U2[4] );
   const double by = 0.5 * ( U1[5] + U2[5] );
   const double bz = 0.5 * ( U1[6] + U2[6] );
   double uu, bb, mml, bbl, mmr, bbr, ptl, ptr, pt, p;
   double a2, a, ca2, ca, c2, ct, cs2, cs, cf2, cf, rr, bp2, sbx;
   double af2, af, as2, as, bty, btz, th1, th2, g21, vb, sgnbt, fcs, fcf;
   int k, deg;
#define LV(a,b) lv[(a)*NF+(b)]
#define RV(a,b) rv[(a)*NF+(b)]
   *neg_pressure = 0;
   if( r <= 0.0 ) return 1;
   uu = u*u + v*v + w*w;
   bb = bx*bx + by*by + bz*bz;
   mml = U1[1]*U1[1] + U1[2]*U1[2] + U1[3]*U1[3];
   bbl = U1[4]*U1[4] + U1[5]*U1[5] + U1[6]*U1[6];
   mmr = U2[1]*U2[1] + U2[2]*U2[2] + U2[3]*U2[3];
   bbr = U2[4]*U2[4] + U2[5]*U2[5] + U2[6]*U2[6];
   ptl = (gm-1.0)*( U1[7] - 0.5*mml/U1[0] - 0.5*bbl ) + 0.5*bbl;
   ptr = (gm-1.0)*( U2[7] - 0.5*mmr/U2[0] - 0.5*bbr ) + 0.5*bbr;
   pt = 0.5 * ( ptl + ptr );
   p = pt - 0.5*bb;
   if( p < 0.0 ){ p = 0.0; *neg_pressure = 1; }

   a2 = gm*p / r;       if( a2 < 0.0 ) a2 = 0.0;
   a = sqrt( a2 );
   ca2 = bx*bx/r;       ca = sqrt( ca2 );
   c2 = 0.5*(bb/r+a2);
   ct = c2*c2-a2*ca2;   if( ct < 0.0 ) ct = 0.0;
   cs2 = c2 - sqrt(ct); if( cs2 < 0.0 ) cs2 = SMALL;
   cs = sqrt( cs2 );
   cf2 = c2 + sqrt(ct); if( cf2 < 0.0 ) cf2 = SMALL;
   cf = sqrt( cf2 );

   rr  = sqrt( r );
   bp2 = by*by + bz*bz;
   sbx = (bx<0.0) ? -1.0 : 1.0;
   deg = (bp2 < SMALL) && (fabs(ca2-a2) < SMALL);      /* degenerate triple point */
   af2 = deg ? 1 : (cf2-ca2) / (cf2-cs2); if( af2 < 0.0 ) af2 = 0.0;
   af  = sqrt( af2 );
   as2 = deg ? 1 : (cf2- a2) / (cf2-cs2); if( as2 < 0.0 ) as2 = 0.0;
   as  = sqrt( as2 );
   bty = bp2 > SMALL ? by / sqrt( bp2 ) : 1.0/sqrt(2.0);
   btz = bp2 > SMALL ? bz / sqrt( bp2 ) : 1.0/sqrt(2.0);
   g21 = (gm-2.0)/(gm-1.0);
   th1 = 1.0 / ( af2*a2*(cf2-g21*a2) + as2*cf2*(cs2-g21*a2) );
   th2 = 1.0 / ( af2*cf*a*sbx + as2*cs*ca*sbx );
   vb  = bty*v+btz*w;

   lam[0] = u - cf; lam[1] = u - ca; lam[2] = u - cs; lam[3] = u;
   lam[4] = u + cs; lam[5] = u + ca; lam[6] = u + cf; lam[7] = 0;

   /* right eigenvectors, one row per characteristic */
   RV(0,0) = af;                  RV(0,1) = af * (u-cf);
   RV(0,2) = af*v + as*bty*ca*sbx; RV(0,3) = af*w + as*btz*ca*sbx;
   RV(0,4) = 0;                   RV(0,5) = as*bty*cf / rr;  RV(0,6) = as*btz*cf / rr;
   RV(0,7) = 0.5*af*uu + af*cf2/(gm-1.0) - af*cf*u + as*ca*sbx*vb + g21*af*(cf2-a2);

   RV(1,0) = 0; RV(1,1) = 0; RV(1,2) = btz*sbx; RV(1,3) = - bty*sbx; RV(1,4) = 0;
   RV(1,5) = btz/rr; RV(1,6) = - bty/rr; RV(1,7) = (btz*v-bty*w)*sbx;

   RV(2,0) = as;                  RV(2,1) = as * (u-cs);
   RV(2,2) = as*v - af*bty*a*sbx; RV(2,3) = as*w - af*btz*a*sbx;
   RV(2,4) = 0;  RV(2,5) = - af*bty*a2 / (cf*rr); RV(2,6) = - af*btz*a2 / (cf*rr);
   RV(2,7) = 0.5*as*uu + as*cs2/(gm-1.0) - as*cs*u - af*a*sbx*vb + g21*as*(cs2-a2);

   RV(3,0) = 1; RV(3,1) = u; RV(3,2) = v; RV(3,3) = w; RV(3,4) = 0; RV(3,5) = 0; RV(3,6) = 0;
   RV(3,7) = 0.5*uu;

   RV(4,0) = as;                  RV(4,1) = as * (u+cs);
   RV(4,2) = as*v + af*bty*a*sbx; RV(4,3) = as*w + af*btz*a*sbx;
   RV(4,4) = 0;  RV(4,5) = - af*bty*a2 / (cf*rr); RV(4,6) = - af*btz*a2 / (cf*rr);
   RV(4,7) = 0.5*as*uu + as*cs2/(gm-1.0) + as*cs*u + af*a*sbx*vb + g21*as*(cs2-a2);

   RV(5,0) = 0; RV(5,1) = 0; RV(5,2) = - btz*sbx; RV(5,3) = + bty*sbx; RV(5,4) = 0;
   RV(5,5) = btz/rr; RV(5,6) = - bty/rr; RV(5,7) = - (btz*v-bty*w)*sbx;

   RV(6,0) = af;                  RV(6,1) = af * (u+cf);
   RV(6,2) = af*v - as*bty*ca*sbx; RV(6,3) = af*w - as*btz*ca*sbx;
   RV(6,4) = 0;                   RV(6,5) = as*bty*cf / rr;  RV(6,6) = as*btz*cf / rr;
   RV(6,7) = 0.5*af*uu + af*cf2/(gm-1.0) + af*cf*u - as*ca*sbx*vb + g21*af*(cf2-a2);

   for( k = 0; k < NF; k++ ){ RV(7,k) = 0; LV(7,k) = 0; }

   /* left eigenvectors */
   LV(0,0) = 0.25*th1*af*a2*uu + 0.5*th2*( af*a*u*sbx - as*cs*vb );
   LV(0,1) = -0.5*th1*af*a2*u - 0.5*th2*af*a*sbx;
   LV(0,2) = -0.5*th1*af*a2*v + 0.5*th2*as*bty*cs;
   LV(0,3) = -0.5*th1*af*a2*w + 0.5*th2*as*btz*cs;
   LV(0,4) = 0;
   LV(0,5) =  0.5*th1*as*bty*cf*rr*(cs2-g21*a2);
   LV(0,6) =  0.5*th1*as*btz*cf*rr*(cs2-g21*a2);
   LV(0,7) =  0.5*th1*af*a2;

   LV(1,0) = -0.5*(btz*v-bty*w)*sbx; LV(1,1) = 0; LV(1,2) = 0.5*btz*sbx; LV(1,3) = -0.5*bty*sbx;
   LV(1,4) = 0; LV(1,5) = 0.5*btz*rr; LV(1,6) = -0.5*bty*rr; LV(1,7) = 0;

   LV(2,0) = 0.25*th1*as*cf2*uu + 0.5*th2*( as*ca*u*sbx + af*cf*vb );
   LV(2,1) = -0.5*th1*as*cf2*u - 0.5*th2*as*ca*sbx;
   LV(2,2) = -0.5*th1*as*cf2*v - 0.5*th2*af*bty*cf;
   LV(2,3) = -0.5*th1*as*cf2*w - 0.5*th2*af*btz*cf;
   LV(2,4) = 0;
   LV(2,5) = -0.5*th1*af*bty*cf*rr*(cf2-g21*a2);
   LV(2,6) = -0.5*th1*af*btz*cf*rr*(cf2-g21*a2);
   LV(2,7) =  0.5*th1*as*cf2;

   LV(3,0) = 1.0 - 0.5*th1*uu*(af2*a2+as2*cf2);
   LV(3,1) =  th1*(af2*a2+as2*cf2)*u;
   LV(3,2) =  th1*(af2*a2+as2*cf2)*v;
   LV(3,3) =  th1*(af2*a2+as2*cf2)*w;
   LV(3,4) = 0;
   LV(3,5) =  th1*af*as*bty*cf*rr*(cf2-cs2);
   LV(3,6) =  th1*af*as*btz*cf*rr*(cf2-cs2);
   LV(3,7) = -th1*(af2*a2+as2*cf2);

   LV(4,0) = 0.25*th1*as*cf2*uu - 0.5*th2*( as*ca*u*sbx + af*cf*vb );
   LV(4,1) = -0.5*th1*as*cf2*u + 0.5*th2*as*ca*sbx;
   LV(4,2) = -0.5*th1*as*cf2*v + 0.5*th2*af*bty*cf;
   LV(4,3) = -0.5*th1*as*cf2*w + 0.5*th2*af*btz*cf;
   LV(4,4) = 0;
   LV(4,5) = -0.5*th1*af*bty*cf*rr*(cf2-g21*a2);
   LV(4,6) = -0.5*th1*af*btz*cf*rr*(cf2-g21*a2);
   LV(4,7) =  0.5*th1*as*cf2;

   LV(5,0) = +0.5*(btz*v-bty*w)*sbx; LV(5,1) = 0; LV(5,2) = -0.5*btz*sbx; LV(5,3) = 0.5*bty*sbx;
   LV(5,4) = 0; LV(5,5) = 0.5*btz*rr; LV(5,6) = -0.5*bty*rr; LV(5,7) = 0;

   LV(6,0) = 0.25*th1*af*a2*uu - 0.5*th2*( af*a*u*sbx - as*cs*vb );
   LV(6,1) = -0.5*th1*af*a2*u + 0.5*th2*af*a*sbx;
   LV(6,2) = -0.5*th1*af*a2*v - 0.5*th2*as*bty*cs;
   LV(6,3) = -0.5*th1*af*a2*w - 0.5*th2*as*btz*cs;
   LV(6,4) = 0;
   LV(6,5) =  0.5*th1*as*bty*cf*rr*(cs2-g21*a2);
   LV(6,6) =  0.5*th1*as*btz*cf*rr*(cs2-g21*a2);
   LV(6,7) =  0.5*th1*af*a2;

   /* continuity of the fast / slow vectors across By = 0 (spatialmethodeno.cpp:554-568) */
   sgnbt = ( (by>0.0) || ( fabs(by) < SMALL && (bz>0.0) ) ) ? 1.0 : -1.0;
   fcs = a2 > ca2 ? sgnbt : 1.0;
   fcf = a2 < ca2 ? sgnbt : 1.0;
   for( k = 0; k < NF; k++ ){
      RV(0,k) *= fcf; RV(6,k) *= fcf; LV(0,k) *= fcf; LV(6,k) *= fcf;
      RV(2,k) *= fcs; RV(4,k) *= fcs; LV(2,k) *= fcs; LV(4,k) *= fcs;
   }
#undef LV
#undef RV
   return 0;
}

/* Swap of the x and y roles within one state / flux vector
   (getEigensG / getNumericalFluxG: components 1<->2 and 4<->5). */
static void swap_xy( double* a ){
   double t = a[1]; a[1] = a[2]; a[2] = t;
   t = a[4]; a[4] = a[5]; a[5] = t;
}

/* ENO-2 candidate selection, spatialmethodenoroe.cpp:240-254 (the same
   rule is used on each LF half in spatialmethodenolf.cpp:294-315). */
static double eno_minus( const double* w, const double* Vw ){
   if( fabs(Vw[0]) < fabs(Vw[1]) ) return -(1.0/2.0)*w[0] + (3.0/2.0)*w[1];
   return (1.0/2.0)*w[1] + (1.0/2.0)*w[2];
}
static double eno_plus( const double* w, const double* Vw ){
   if( fabs(Vw[1]) < fabs(Vw[2]) ) return (1.0/2.0)*w[1] + (1.0/2.0)*w[2];
   return (3.0/2.0)*w[2] - (1.0/2.0)*w[3];
}

/* One ENO-Roe interface, x frame: spatialmethodenoroe.cpp:182-282.
   Fs[m][l], l = 0..3 <-> cells i-1..i+2; Vs[m][l], l = 0..2 <-> i-1..i+1. */
static int flux_roe( double gm, const double* U1, const double* U2, double Fs[NF][4],
                     double Vs[NF][3], double* Fn, double* lam, double* LU, double* smax,
                     int* negp )
{
   double lv[NF*NF], rv[NF*NF], w[4], Vw[3], fw[NF];
   int k, l, m;
   if( orc_eigens_f( gm, U1, U2, lam, lv, rv, negp ) ) return 1;
   *smax = 0.0;
   for( k = 0; k < NF; k++ ){ double s = fabs( lam[k] ); if( s > *smax ) *smax = s; }
   for( k = 0; k < NF; k++ ){
      double wm, wp;
      for( l = 0; l < 4; l++ ){ w[l] = 0.0; for( m = 0; m < NF; m++ ) w[l] += lv[k*NF+m]*Fs[m][l]; }
      for( l = 0; l < 3; l++ ){ Vw[l] = 0.0; for( m = 0; m < NF; m++ ) Vw[l] += lv[k*NF+m]*Vs[m][l]; }
      wm = eno_minus( w, Vw );
      wp = eno_plus( w, Vw );
      if( lam[k] >= 0 && wm < 1.0e10 )      fw[k] = wm;   /* upwind, no entropy fix */
      else if( lam[k] <= 0 && wp < 1.0e10 ) fw[k] = wp;
      else                                  fw[k] = 0.0;
   }
   for( m = 0; m < NF; m++ ){ Fn[m] = 0.0; for( k = 0; k < NF; k++ ) Fn[m] += rv[k*NF+m]*fw[k]; }
   for( k = 0; k < NF; k++ ){ LU[k] = 0.0; for( m = 0; m < NF; m++ ) LU[k] += lv[k*NF+m]*U1[m]; }
   return 0;
}

/* One ENO-LF interface, x frame: spatialmethodenolf.cpp:233-336. */
static int flux_lf( double gm, const double* U1, const double* U2, double Us[NF][4],
                    double Fs[NF][4], const double* alpha, double* Fn, double* lam, double* LU,
                    double* smax, int* negp )
{
   double lv[NF*NF], rv[NF*NF], RU[4], RF[4], w[4], Vw[3], fw[NF];
   int k, l, m;
   if( orc_eigens_f( gm, U1, U2, lam, lv, rv, negp ) ) return 1;
   *smax = 0.0;
   for( k = 0; k < NF; k++ ){ double s = fabs( lam[k] ); if( s > *smax ) *smax = s; }
   for( k = 0; k < NF; k++ ){
      double wm, wp;
      for( l = 0; l < 4; l++ ){
         RU[l] = 0.0; RF[l] = 0.0;
         for( m = 0; m < NF; m++ ){ RU[l] += lv[k*NF+m]*Us[m][l]; RF[l] += lv[k*NF+m]*Fs[m][l]; }
      }
      for( l = 0; l < 4; l++ ) w[l] = 0.5*( RF[l] + alpha[k]*RU[l] );
      for( l = 0; l < 3; l++ ) Vw[l] = w[l+1] - w[l];
      wm = eno_minus( w, Vw );
      for( l = 0; l < 4; l++ ) w[l] = 0.5*( RF[l] - alpha[k]*RU[l] );
      for( l = 0; l < 3; l++ ) Vw[l] = w[l+1] - w[l];
      wp = eno_plus( w, Vw );
      fw[k] = wm + wp;
      LU[k] = RU[1];
   }
   for( m = 0; m < NF; m++ ){ Fn[m] = 0.0; for( k = 0; k < NF; k++ ) Fn[m] += rv[k*NF+m]*fw[k]; }
   return 0;
}

/* ENO-LF dissipation coefficients, spatialmethodenolf.cpp:66-125: per-row
   (alphaF[k][j], max over i) and per-column (alphaG[k][i], max over j)
   maxima of |lambda_k| over i in [1, nx+2), j in [1, ny+2), skipping the
   (i < 2 && j < 2) corner. */
static int lf_alpha( orc_ctx* c, const double* U, int* negp )
{
   int i, j, k, np;
   double s[NF], lam[NF];
   if( c->alpha_fixed ) return 0;
   for( k = 0; k < NF; k++ ){
      for( i = 1; i < c->nx+2; i++ ) c->aG[(size_t)k*c->NX+i] = 0.0;
      for( j = 1; j < c->ny+2; j++ ) c->aF[(size_t)k*c->NY+j] = 0.0;
   }
   for( i = 1; i < c->nx+2; i++ ) for( j = 1; j < c->ny+2; j++ ){
      if( i < 2 && j < 2 ) continue;
      for( k = 0; k < NF; k++ ) s[k] = AT(U,k,i,j);
      if( orc_eigenvalues_at( c->gamma, s, lam, &np ) ) return 1;
      *negp = np;
      for( k = 0; k < NF; k++ ){ double a = fabs(lam[k]); if( a > c->aF[(size_t)k*c->NY+j] ) c->aF[(size_t)k*c->NY+j] = a; }
      swap_xy( s );
      if( orc_eigenvalues_at( c->gamma, s, lam, &np ) ) return 1;
      *negp = np;
      for( k = 0; k < NF; k++ ){ double a = fabs(lam[k]); if( a > c->aG[(size_t)k*c->NX+i] ) c->aG[(size_t)k*c->NX+i] = a; }
   }
   return 0;
}

/* Test hook: the dissipation coefficients of a whole grid (lf_alpha over a
   grid of nx x ny cells whose ghost layers are already filled), computed
   without a context, so that a window of a large grid can be integrated
   with the coefficients of the whole grid (orc_set_lf_alpha). */
int orc_lf_alpha_grid( double gamma, int nx, int ny, const double* U, double* aF, double* aG )
{
   orc_ctx c0;
   int negp = 0;
   memset( &c0, 0, sizeof c0 );
   c0.nx = nx; c0.ny = ny; c0.NX = nx+4; c0.NY = ny+4; c0.gamma = gamma;
   c0.aF = aF; c0.aG = aG;
   return lf_alpha( &c0, U, &negp ) ? ORC_ERR_NEGATIVE_DENSITY : ORC_OK;
}

/* Test hook: fix aF [8][NY] and aG [8][NX] for the following ENO-LF
   integrations of this context (NULL returns to computing them). */
void orc_set_lf_alpha( orc_ctx* c, const double* aF, const double* aG )
{
   if( !aF || !aG ){ c->alpha_fixed = 0; return; }
   memcpy( c->aF, aF, (size_t)NF*c->NY*sizeof(double) );
   memcpy( c->aG, aG, (size_t)NF*c->NX*sizeof(double) );
   c->alpha_fixed = 1;
}

/* SpatialMethodEnoRoe::integrate (spatialmethodenoroe.cpp:33-179) and
   SpatialMethodEnoLF::integrate (spatialmethodenolf.cpp:33-230).
   The returned status follows the reference: the status of the last
   interface evaluated (so a clamped pressure there reports
   ErrorNegativePressure without isError). */
/* std::max({ a, ... }) over the 8 signed wave speeds: the first largest,
   so a NaN candidate never replaces the running value. */
static double max_speeds( double m, double u, double cf, double ca, double cs )
{
   const double v[7] = { u - cf, u - ca, u - cs, u, u + cs, u + ca, u + cf };
   int n;
   for( n = 0; n < 7; n++ ) if( m < v[n] ) m = v[n];
   return m;
}

/* SpatialMethodCentralFD2::integrate (spatialmethodcentralfd2.cpp:44-160):
   physical fluxes on the interior and the ring of ghost cells around it,
   the four ring corners skipped with nxFirst / nxLast for both indices
   (lines 60-64); the maxima of the signed wave speeds (not |lambda|) for
   dtIdeal; UL from central differences of F and G.  A non-positive density
   returns at the first such cell in loop order before UL is formed; a
   non-positive pressure is fatal too, reported at the last such cell, after
   UL and dtIdeal.  F and G of skipped cells keep their initial zeros (the
   reference leaves them unset). */
static int cfd_integrate( orc_ctx* c, double* U, double* UL, double* dtIdeal, int* is_error )
{
   const int nx = c->nx, ny = c->ny, f0 = 2, l0 = nx + 2;
   const double gm = c->gamma;
   double cxm = 0.0, cym = 0.0;
   int pok = 1, i, j, k, st;

   st = orc_apply_bc( c, U, is_error );
   if( *is_error ) return st;
   for( i = f0-1; i < nx+3; i++ ) for( j = f0-1; j < ny+3; j++ ){
      double r, mx, my, mz, bx, by, bz, e, u, v, w, uu, ub, bb, p, pt;
      double c2, ca2, ca, ct2, ctemp, cs2, cs, cf2, cf;
      if( ( i < f0 && j < f0 ) || ( i < f0 && j >= l0 ) || ( i >= l0 && j < f0 ) ||
          ( i >= l0 && j >= l0 ) ) continue;
      r = AT(U,0,i,j);
      mx = AT(U,1,i,j); u = mx / r;
      my = AT(U,2,i,j); v = my / r;
      mz = AT(U,3,i,j); w = mz / r;
      bx = AT(U,4,i,j); by = AT(U,5,i,j); bz = AT(U,6,i,j); e = AT(U,7,i,j);
      uu = u*u + v*v + w*w;
      ub = u*bx + v*by + w*bz;
      bb = bx*bx + by*by + bz*bz;
      p = (gm-1.0)*(e-0.5*r*uu-0.5*bb);
      pt = p + 0.5*bb;
      if( r <= 0.0 ){
         c->cfd_i = i; c->cfd_j = j;
         *is_error = 1;
         return ORC_ERR_NEGATIVE_DENSITY;
      }
      if( p <= 0.0 ){ pok = 0; c->cfd_i = i; c->cfd_j = j; }
      AT(c->F,0,i,j) = mx;
      AT(c->F,1,i,j) = mx*u - bx*bx + pt;
      AT(c->F,2,i,j) = my*u - bx*by;
      AT(c->F,3,i,j) = mz*u - bx*bz;
      AT(c->F,4,i,j) = 0;
      AT(c->F,5,i,j) = by*u - bx*v;
      AT(c->F,6,i,j) = bz*u - bx*w;
      AT(c->F,7,i,j) = (e+pt)*u - bx*ub;
      AT(c->G,0,i,j) = my;
      AT(c->G,1,i,j) = mx*v - by*bx;
      AT(c->G,2,i,j) = my*v - by*by + pt;
      AT(c->G,3,i,j) = mz*v - by*bz;
      AT(c->G,4,i,j) = bx*v - by*u;
      AT(c->G,5,i,j) = 0;
      AT(c->G,6,i,j) = bz*v - by*w;
      AT(c->G,7,i,j) = (e+pt)*v - by*ub;
      c2 = gm*p / r; if( c2 < 0.0 ) c2 = 0.0;
      ca2 = bx*bx/r;
      ca = sqrt(ca2);
      ct2 = 0.5*(bb/r+c2);
      ctemp = ct2*ct2-c2*ca2; if( ctemp < 0.0 ) ctemp = 0.0;
      cs2 = ct2 - sqrt(ctemp); if( cs2 < 0.0 ) cs2 = 0.0;
      cs = sqrt(cs2);
      cf2 = ct2 + sqrt(ctemp); if( cf2 < 0.0 ) cf2 = 0.0;
      cf = sqrt(cf2);
      cxm = max_speeds( cxm, u, cf, ca, cs );
      ca2 = by*by/r;
      ca = sqrt(ca2);
      ct2 = 0.5*(bb/r+c2);
      ctemp = ct2*ct2-c2*ca2; if( ctemp < 0.0 ) ctemp = 0.0;
      cs2 = ct2 - sqrt(ctemp); if( cs2 < 0.0 ) cs2 = 0.0;
      cs = sqrt(cs2);
      cf2 = ct2 + sqrt(ctemp); if( cf2 < 0.0 ) cf2 = 0.0;
      cf = sqrt(cf2);
      cym = max_speeds( cym, v, cf, ca, cs );
   }
   {  /* std::min( dx/cxmax, dy/cymax ) */
      const double ax = c->dx/cxm, ay = c->dy/cym;
      *dtIdeal = ( ay < ax ) ? ay : ax;
   }
   for( k = 0; k < NF; k++ ) for( i = 2; i < nx+2; i++ ) for( j = 2; j < ny+2; j++ )
      AT(UL,k,i,j) = -(1.0/(2.0*c->dx)) * ( AT(c->F,k,i+1,j) - AT(c->F,k,i-1,j) )
                     -(1.0/(2.0*c->dy)) * ( AT(c->G,k,i,j+1) - AT(c->G,k,i,j-1) );
   if( !pok ){ *is_error = 1; return ORC_ERR_NEGATIVE_PRESSURE; }
   *is_error = 0;
   return ORC_OK;
}

int orc_integrate( orc_ctx* c, double* U, double* UL, double* dtIdeal, int* is_error )
{
   const int nx = c->nx, ny = c->ny, lf = (c->scheme == 3);
   double U1[NF], U2[NF], Us[NF][4], Fs[NF][4], Vs[NF][3], Fn[NF], lam[NF], LU[NF], al[NF];
   double mX = 0.0, mY = 0.0, s;
   int i, j, k, l, st, negp = 0;

   if( c->scheme == 1 ) return cfd_integrate( c, U, UL, dtIdeal, is_error );

   st = orc_apply_bc( c, U, is_error );
   if( *is_error ) return st;
   fluxes( c, U );
   if( !lf ){
      for( k = 0; k < NF; k++ ) for( i = 0; i < nx+3; i++ ) for( j = 0; j < ny+3; j++ ){
         AT(c->VF,k,i,j) = AT(c->F,k,i+1,j) - AT(c->F,k,i,j);
         AT(c->VG,k,i,j) = AT(c->G,k,i,j+1) - AT(c->G,k,i,j);
      }
   } else {
      if( lf_alpha( c, U, &negp ) ){ *is_error = 1; return ORC_ERR_NEGATIVE_DENSITY; }
   }

   /* x interfaces i+1/2, i in [1, nx+2), j in [2, ny+2) */
   for( i = 1; i < nx+2; i++ ) for( j = 2; j < ny+2; j++ ){
      for( k = 0; k < NF; k++ ){
         U1[k] = ( c->bc[L] == OPN && i < 2 ) ? AT(U,k,i+1,j) : AT(U,k,i,j);
         U2[k] = ( c->bc[R] == OPN && i > nx ) ? AT(U,k,i,j) : AT(U,k,i+1,j);
         for( l = 0; l < 4; l++ ){ Us[k][l] = AT(U,k,i-1+l,j); Fs[k][l] = AT(c->F,k,i-1+l,j); }
         if( !lf ) for( l = 0; l < 3; l++ ) Vs[k][l] = AT(c->VF,k,i-1+l,j);
         al[k] = c->aF[(size_t)k*c->NY+j];
      }
      if( lf ? flux_lf( c->gamma, U1, U2, Us, Fs, al, Fn, lam, LU, &s, &negp )
             : flux_roe( c->gamma, U1, U2, Fs, Vs, Fn, lam, LU, &s, &negp ) ){
         *is_error = 1; return ORC_ERR_NEGATIVE_DENSITY;
      }
      for( k = 0; k < NF; k++ ){ AT(c->FN,k,i,j) = Fn[k]; AT(c->cx,k,i,j) = lam[k]; AT(c->LUx,k,i,j) = LU[k]; }
      if( s > mX ) mX = s;
   }
   /* y interfaces j+1/2, i in [2, nx+2), j in [1, ny+2); x/y roles swapped */
   for( i = 2; i < nx+2; i++ ) for( j = 1; j < ny+2; j++ ){
      double t;
      for( k = 0; k < NF; k++ ){
         U1[k] = ( c->bc[B] == OPN && j < 2 ) ? AT(U,k,i,j+1) : AT(U,k,i,j);
         U2[k] = ( c->bc[T] == OPN && j > ny ) ? AT(U,k,i,j) : AT(U,k,i,j+1);
         for( l = 0; l < 4; l++ ){ Us[k][l] = AT(U,k,i,j-1+l); Fs[k][l] = AT(c->G,k,i,j-1+l); }
         if( !lf ) for( l = 0; l < 3; l++ ) Vs[k][l] = AT(c->VG,k,i,j-1+l);
         al[k] = c->aG[(size_t)k*c->NX+i];
      }
      swap_xy( U1 ); swap_xy( U2 );
      for( l = 0; l < 4; l++ ){
         t = Us[1][l]; Us[1][l] = Us[2][l]; Us[2][l] = t; t = Us[4][l]; Us[4][l] = Us[5][l]; Us[5][l] = t;
         t = Fs[1][l]; Fs[1][l] = Fs[2][l]; Fs[2][l] = t; t = Fs[4][l]; Fs[4][l] = Fs[5][l]; Fs[5][l] = t;
      }
      for( l = 0; l < 3; l++ ){
         t = Vs[1][l]; Vs[1][l] = Vs[2][l]; Vs[2][l] = t; t = Vs[4][l]; Vs[4][l] = Vs[5][l]; Vs[5][l] = t;
      }
      negp = 0;
      if( lf ? flux_lf( c->gamma, U1, U2, Us, Fs, al, Fn, lam, LU, &s, &negp )
             : flux_roe( c->gamma, U1, U2, Fs, Vs, Fn, lam, LU, &s, &negp ) ){
         *is_error = 1; return ORC_ERR_NEGATIVE_DENSITY;
      }
      swap_xy( Fn );
      for( k = 0; k < NF; k++ ){ AT(c->GN,k,i,j) = Fn[k]; AT(c->cy,k,i,j) = lam[k]; AT(c->LUy,k,i,j) = LU[k]; }
      if( s > mY ) mY = s;
   }
   {  /* std::min semantics: returns the first argument unless the second is smaller */
      const double ax = c->dx/mX, ay = c->dy/mY;
      *dtIdeal = ( ay < ax ) ? ay : ax;
   }
   for( k = 0; k < NF; k++ ) for( i = 2; i < nx+2; i++ ) for( j = 2; j < ny+2; j++ )
      AT(UL,k,i,j) = -(1.0/c->dx)*( AT(c->FN,k,i,j) - AT(c->FN,k,i-1,j) )
                     -(1.0/c->dy)*( AT(c->GN,k,i,j) - AT(c->GN,k,i,j-1) );
   *is_error = 0;
   return negp ? ORC_ERR_NEGATIVE_PRESSURE : ORC_OK;
}

void orc_get_characteristics( const orc_ctx* c, double* cx, double* cy, double* LUx, double* LUy )
{
   const size_t tot = (size_t)NF*c->NX*c->NY*sizeof(double);
   if( cx ) memcpy( cx, c->cx, tot );
   if( cy ) memcpy( cy, c->cy, tot );
   if( LUx ) memcpy( LUx, c->LUx, tot );
   if( LUy ) memcpy( LUy, c->LUy, tot );
}

/* timeintegrationmethod.cpp:35-90 */
int orc_update_dt( double dt_min, double dt_max, double cfl, double* dt_inout, double ideal,
                   int* is_error )
{
   double dt = *dt_inout;
   *is_error = 0;
   if( cfl == 0.0 ) return ORC_NO_CHANGE;
   while( dt < 0.5*cfl*ideal ) dt *= 2.0;
   while( dt > cfl*ideal ) dt /= 2.0;
   if( dt > dt_max ) dt = dt_max;
   if( dt < dt_min ){ *is_error = 1; return ORC_ERR_TIME_UNDERFLOW; }
   if( dt == *dt_inout ) return ORC_NO_CHANGE;
   *dt_inout = dt;
   return ORC_UPDATED;
}

/* TimeIntegrationRK3::step (timeintegrationrk3.cpp:48-156) including the
   retry: a stage that asks for a smaller dt restarts from U1 = U + dt*UL
   with UL still holding the last stage's L(U).  The dead borderFlux blend
   is not restated.  TimeIntegrationEuler::step: timeintegrationeuler.cpp:26-64. */
int orc_step( orc_ctx* c, double* U, double* dt_inout, int* is_error )
{
   const int nx = c->nx, ny = c->ny;
   double ideal = 0.0, dt = *dt_inout;
   int st, k, i, j;
   st = orc_integrate( c, U, c->UL, &ideal, is_error );
   if( *is_error ) return st;
   if( c->time_method == 1 ){
      st = orc_update_dt( c->dt_min, c->dt_max, c->cfl, &dt, ideal, is_error );
      if( *is_error ) return st;
      for( k = 0; k < NF; k++ ) for( i = 2; i < nx+2; i++ ) for( j = 2; j < ny+2; j++ )
         AT(U,k,i,j) = AT(U,k,i,j) + dt*AT(c->UL,k,i,j);
      *dt_inout = dt;
      return ORC_OK;
   } else {
      double d1 = *dt_inout, d2 = c->dt_max, d3 = c->dt_max;
      st = orc_update_dt( c->dt_min, c->dt_max, c->cfl, &d1, ideal, is_error );
      if( *is_error ) return st;
      for( ;; ){
         dt = d1 < d2 ? d1 : d2;   /* std::min of an initializer list: the first smallest */
         if( d3 < dt ) dt = d3;
         for( k = 0; k < NF; k++ ) for( i = 2; i < nx+2; i++ ) for( j = 2; j < ny+2; j++ )
            AT(c->U1,k,i,j) = AT(U,k,i,j) + dt*AT(c->UL,k,i,j);
         st = orc_integrate( c, c->U1, c->UL, &ideal, is_error );
         if( *is_error ) return st;
         st = orc_update_dt( c->dt_min, c->dt_max, c->cfl, &d2, ideal, is_error );
         if( *is_error ) return st;
         if( d2 < dt ){ c->retries++; continue; }
         for( k = 0; k < NF; k++ ) for( i = 2; i < nx+2; i++ ) for( j = 2; j < ny+2; j++ )
            AT(c->U2,k,i,j) = (3.0/4.0)*AT(U,k,i,j) + (1.0/4.0)*AT(c->U1,k,i,j)
                            + (1.0/4.0)*dt*AT(c->UL,k,i,j);
         st = orc_integrate( c, c->U2, c->UL, &ideal, is_error );
         if( *is_error ) return st;
         st = orc_update_dt( c->dt_min, c->dt_max, c->cfl, &d3, ideal, is_error );
         if( *is_error ) return st;
         if( d3 < dt ){ c->retries++; continue; }
         for( k = 0; k < NF; k++ ) for( i = 2; i < nx+2; i++ ) for( j = 2; j < ny+2; j++ )
            AT(U,k,i,j) = (1.0/3.0)*AT(U,k,i,j) + (2.0/3.0)*AT(c->U2,k,i,j)
                        + (2.0/3.0)*dt*AT(c->UL,k,i,j);
         break;
      }
      *dt_inout = dt;
      *is_error = 0;
      return ORC_OK;
   }
}

/* Interior range of the div B stencils: one cell in from every
   non-periodic side (div_b_fix.cpp:17-101, 161-245), and the periodic
   wrap of the Bx, By ghost layers. */
static void divb_prepare( orc_ctx* c, double* U, int* x0, int* x1, int* y0, int* y1 )
{
   const int f = 2, lx = c->nx+2, ly = c->ny+2;
   int k, i, j;
   *x0 = f; *x1 = lx; *y0 = f; *y1 = ly;
   if( c->bc[L] == PER ){ for( k = 4; k <= 5; k++ ) for( j = f; j < ly; j++ ){ AT(U,k,f-2,j) = AT(U,k,lx-2,j); AT(U,k,f-1,j) = AT(U,k,lx-1,j); } }
   else *x0 = f+1;
   if( c->bc[R] == PER ){ for( k = 4; k <= 5; k++ ) for( j = f; j < ly; j++ ){ AT(U,k,lx,j) = AT(U,k,f,j); AT(U,k,lx+1,j) = AT(U,k,f+1,j); } }
   else *x1 = lx-1;
   if( c->bc[B] == PER ){ for( k = 4; k <= 5; k++ ) for( i = f; i < lx; i++ ){ AT(U,k,i,f-2) = AT(U,k,i,ly-2); AT(U,k,i,f-1) = AT(U,k,i,ly-1); } }
   else *y0 = f+1;
   if( c->bc[T] == PER ){ for( k = 4; k <= 5; k++ ) for( i = f; i < lx; i++ ){ AT(U,k,i,ly) = AT(U,k,i,f); AT(U,k,i,ly+1) = AT(U,k,i,f+1); } }
   else *y1 = ly-1;
}

/* div_b_fix.cpp:4-126 */
void orc_divb_calc( orc_ctx* c, double* U, double* maxdivb, double* totdivb )
{
   int x0, x1, y0, y1, i, j;
   double mx = 0.0, tot = 0.0;
   divb_prepare( c, U, &x0, &x1, &y0, &y1 );
   for( i = x0; i < x1; i++ ) for( j = y0; j < y1; j++ ){
      const double d = fabs( (AT(U,4,i+1,j)-AT(U,4,i-1,j))/(2.0*c->dx)
                           + (AT(U,5,i,j+1)-AT(U,5,i,j-1))/(2.0*c->dy) );
      if( d > mx ) mx = d;
      tot += d;
   }
   *maxdivb = mx;
   *totdivb = tot*(c->dx*c->dy);
}

/* Potential boundary fill after each sweep (div_b_fix.cpp:282-364):
   periodic wraps both ghost layers, open copies the edge into the first
   ghost layer, Dirichlet / Neumann leave the ghosts alone. */
static void phi_bc( orc_ctx* c )
{
   const int f = 2, lx = c->nx+2, ly = c->ny+2;
   int i, j;
   if( c->bc[L] == PER ) for( j = f; j < ly; j++ ){ PHI(f-2,j) = PHI(lx-2,j); PHI(f-1,j) = PHI(lx-1,j); }
   else if( c->bc[L] == OPN ) for( j = f; j < ly; j++ ) PHI(f-1,j) = PHI(f,j);
   if( c->bc[R] == PER ) for( j = f; j < ly; j++ ){ PHI(lx,j) = PHI(f,j); PHI(lx+1,j) = PHI(f+1,j); }
   else if( c->bc[R] == OPN ) for( j = f; j < ly; j++ ) PHI(lx,j) = PHI(lx-1,j);
   if( c->bc[B] == PER ) for( i = f; i < lx; i++ ){ PHI(i,f-2) = PHI(i,ly-2); PHI(i,f-1) = PHI(i,ly-1); }
   else if( c->bc[B] == OPN ) for( i = f; i < lx; i++ ) PHI(i,f-1) = PHI(i,f);
   if( c->bc[T] == PER ) for( i = f; i < lx; i++ ){ PHI(i,ly) = PHI(i,f); PHI(i,ly+1) = PHI(i,f+1); }
   else if( c->bc[T] == OPN ) for( i = f; i < lx; i++ ) PHI(i,ly) = PHI(i,ly-1);
}

/* div_b_fix.cpp:129-403.  Gauss-Seidel/SOR on the wide (stride-2)
   Laplacian  phi <- phi + omega*(coef*(px*(phi[i+2]+phi[i-2]) +
   py*(phi[j+2]+phi[j-2]) + 2*dBx/dx + 2*dBy/dy) - phi); converged when the
   largest unrelaxed update over the largest |phi| drops to rmax; then
   B += central gradient of phi over the interior plus one ring. */
int orc_divb_sor( orc_ctx* c, const orc_sor_params* sp, double* U, int red_black,
                  int* sweeps, int* is_error )
{
   const double bxf = 4.0/(2.0*c->dx), byf = 4.0/(2.0*c->dy);
   const double pxf = 1.0/(c->dx*c->dx), pyf = 1.0/(c->dy*c->dy);
   const double coef = 1.0/(2*(pxf+pyf));
   double omega, rmax = 0.0, pmax = 0.0;
   int x0, x1, y0, y1, i, j, step, pass, done = 0;
   divb_prepare( c, U, &x0, &x1, &y0, &y1 );
   if( sp->omega_use_static ) omega = sp->omega;
   else {
      const double t = cos(c->dx)+cos(c->dy);
      omega = (8.0-sqrt(64.0-16.0*t*t))/(t*t);
   }
   for( step = 0; step < sp->sor_rsteps; step++ ){
      rmax = 0.0; pmax = 0.0;
      for( pass = 0; pass < (red_black ? 2 : 1); pass++ ){
         for( i = x0; i < x1; i++ ) for( j = y0; j < y1; j++ ){
            double r;
            if( red_black && (((i>>1)+(j>>1))&1) != pass ) continue;
            r  = pxf*( PHI(i+2,j) + PHI(i-2,j) );
            r += pyf*( PHI(i,j+2) + PHI(i,j-2) );
            r += bxf*( AT(U,4,i+1,j) - AT(U,4,i-1,j) );
            r += byf*( AT(U,5,i,j+1) - AT(U,5,i,j-1) );
            r *= coef;
            r -= PHI(i,j);
            PHI(i,j) += omega*r;
            if( fabs(r) > rmax ) rmax = fabs(r);
            if( fabs(PHI(i,j)) > pmax ) pmax = fabs(PHI(i,j));
         }
         /* Red-black: refresh the ghost copies after each colour.  With
            periodic sides the ghosts mirror points of the other colour, and
            one refresh per sweep would feed the second colour stale values
            across the seam (that mixed ordering diverges for omega >= 1.5). */
         if( red_black && pass == 0 ) phi_bc( c );
      }
      phi_bc( c );
      if( rmax/pmax <= sp->sor_rmax ){ done = 1; break; }
   }
   *sweeps = done ? step+1 : step;
   /* The verdict after the loop is the negated test (div_b_fix.cpp:387):
      a NaN ratio (diverged potential, or no sweep at all) counts as
      converged and the correction is applied. */
   if( rmax/pmax > sp->sor_rmax ){ *is_error = 1; return ORC_ERR_NOT_CONVERGED; }
   for( i = x0-1; i < x1+1; i++ ) for( j = y0-1; j < y1+1; j++ ){
      AT(U,4,i,j) += ( PHI(i+1,j) - PHI(i-1,j) )*(1.0/(2.0*c->dx));
      AT(U,5,i,j) += ( PHI(i,j+1) - PHI(i,j-1) )*(1.0/(2.0*c->dy));
   }
   *is_error = 0;
   return ORC_OK;
}

long long orc_retries( const orc_ctx* c ){ return c->retries; }

/* main.cpp:174-344 without output (see ref_harness.cpp: ref_run). */
int orc_run( orc_ctx* c, int nsteps, double t_max, const orc_sor_params* sor, int red_black,
             double* U, double* dt_inout, double* t_inout, int* steps_done,
             double* dt_hist, double* divb_hist, int hist_len, int* is_error )
{
   double dt = *dt_inout, t = *t_inout;
   int step = 1, done = 0, st = ORC_OK, it, sw, e2;
   *is_error = 0;
   orc_init_dirichlet( c, U );
   while( !done ){
      double dmax = -1.0, dsum = 0.0;
      st = orc_step( c, U, &dt, is_error );
      if( st == ORC_ERR_TIME_UNDERFLOW || *is_error ) break;
      if( sor && sor->sor_steps > 0 && step % sor->divb_skip_steps == 0 ){
         for( it = 0; it < sor->sor_steps; it++ ){
            orc_divb_calc( c, U, &dmax, &dsum );
            if( dmax < sor->sor_divbmax ) break;
            if( orc_divb_sor( c, sor, U, red_black, &sw, &e2 ) == ORC_ERR_NOT_CONVERGED ) break;
         }
         orc_divb_calc( c, U, &dmax, &dsum );
      }
      t += dt;
      if( dt_hist && step <= hist_len ) dt_hist[step-1] = dt;
      if( divb_hist && step <= hist_len ) divb_hist[step-1] = dmax;
      if( nsteps > 0 && step == nsteps ) done = 1;
      if( t_max > 0.0 && t >= t_max ) done = 1;
      if( isnan( AT(U,0,2,2) ) ) done = 1;
      step++;
   }
   *dt_inout = dt; *t_inout = t; *steps_done = step-1;
   return st;
}
