/*
 * SimParams3D — the parameter block of the single-partition MLS-MPM step.
 *
 * The non-static fields are declared in the same order and with the same C
 * types as the reference's struct (simulation/parameters_sim_3d.h:40-90), so a
 * caller that already holds a reference SimParams3D can pass its address to
 * the entry points of icempm_b200.h unchanged: both are standard-layout
 * structs with natural alignment, hence byte-identical.
 *
 * The reference's static constants (parameters_sim_3d.h:24-38: pi, dim,
 * nGridArrays and the row indices of the particle SoA) are given here as
 * macros/enum values because C structs cannot hold them.
 */
#ifndef ICEMPM_SIM_PARAMS_3D_H
#define ICEMPM_SIM_PARAMS_3D_H

#ifdef __cplusplus
extern "C" {
#endif

/* Row indices of the particle structure-of-arrays (parameters_sim_3d.h:29-38).
 * Row k of a host buffer with row stride `pitch` holds field k of every
 * particle: soa[k*pitch + i]. */
enum {
    MPM_IDX_UTILITY = 0,   /* int64 status word, bit-cast into a double       */
    MPM_IDX_P       = 1,   /* trial pressure p_tr (written on record steps)   */
    MPM_IDX_Q       = 2,   /* trial deviatoric q_tr (written on record steps) */
    MPM_IDX_JP_INV  = 3,   /* plastic volume ratio tracker Jp_inv             */
    MPM_POSX        = 4,   /* x, y, z                                        */
    MPM_VELX        = 7,   /* vx, vy, vz                                     */
    MPM_FE00        = 10,  /* elastic deformation gradient, row-major 3x3     */
    MPM_BP00        = 19,  /* APIC affine matrix C ("Bp"), row-major 3x3      */
    MPM_N_PTS_ARRAYS = 28
};

/* Status bits of the utility word (mpm_kernels.cuh:13-15; grain id = low 16
 * bits, partition id = bits 24..31, proxypoint3d.cpp:89-110,151-156). */
#define MPM_STATUS_CRUSHED  0x10000LL
#define MPM_STATUS_DISABLED 0x20000LL
#define MPM_STATUS_LIQUID   0x40000LL

#define MPM_PI 3.14159265358979323846
#define MPM_N_GRID_ARRAYS 4

typedef struct SimParams3D
{
    int SetupType;            /* 0 horizontal indentation; 1 cone; 2 tank */

    int nPtsTotal;
    int GridXTotal, GridY, GridZ;
    int IndenterSubdivisions;
    double DomainDimensionX;

    double InitialTimeStep, SimulationEndTime;
    double SimulationTime;
    int UpdateEveryNthStep;
    int SnapshotPeriod;
    int SimulationStep;

    double Gravity, Density, WaterDensity, PoissonsRatio, YoungsModulus;
    double DragGlobal;
    double lambda, mu, kappa;

    double IceCompressiveStrength, IceTensileStrength, IceShearStrength, IceTensileStrength2;
    double NACC_beta;
    double DP_tan_phi, DP_threshold_p;
    double GrainVariability;

    double IndDiameter, IndRSq, IndVelocity, IndDepth;

    double cellsize;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double BlockCutout[3];

    double ParticleVolume, ParticleMass, ParticleViewSize, LiquidParticleMass;

    double indenter_x, indenter_x_initial, indenter_y, indenter_y_initial;
    double Volume;

    int nPartitions;
    int GridHaloSize;
    int PointTransferFrequency;
    int VectorCapacity_transfer;
    double ExtraSpaceForIncomingPoints;
    double PointsTransferBufferFraction;
    double RebalanceThresholdFreeSpaceRemaining;
    double RebalanceThresholdDisabledPercentage;

    double dt_vol_Dpinv, dt_Gravity, vmax, vmax_squared;
    int gbOffset;
    double cellsize_inv, Dp_inv;
    int tpb_P2G, tpb_Upd, tpb_G2P;
    double animation_threshold_pos;
} SimParams3D;

#ifdef __cplusplus
}
#endif

#endif /* ICEMPM_SIM_PARAMS_3D_H */
