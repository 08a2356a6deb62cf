*KEYWORD_ID
g_freesurf
*DIRECTORY
out
*PARAMETERS
accelGravity 9.8
radBoltzmann 5.67e-08
ambientTemp 300.0
ambientPres 101000.0
gasConstant 8.314
*SCALAR_OUT
temp
uvel
vvel
wvel
zr
tempr
*CONTROL_TERMINATION
$ total_time max_iter nonlin_tolerance
  3.5000000000000004e-05 20 1e-05
*CONTROL_TIMESTEP
$ sim_timestep output_timestep
  1e-05 1.0
*GAUSS_LASER_PARAMETERS
$ power absorb radius factor
  250.0 0.35 5e-05 2.0
*MATERIAL_PROPERTIES
$ dens denl viscos tsolid tliquid hsmelt hlfriz
  7800.0 7800.0 0.006 1563.0 1623.0 781501.2214845 1089001.2683744999
$ acpa acpb acpl
  1e-06 500.0 750.0
$ thconsa thconsb thconsc thconla thconlb
  0.0 0.015 15.0 0.015 15.0
*UNDER_RELAXATION
$ urfu urfv urfw urfp urfh
  0.7 0.7 0.7 0.7 0.7
*BOUNDARY_TEMPERATURES
$ west east north bottom preheat
  300.0 300.0 300.0 300.0 300.0
*BOUNDARY_ENERGY_EQUATION
$ htci htcj htckl htckn emiss
  10.0 10.0 10.0 10.0 0.4
*BOUNDARY_MOMENTUM_EQUATION
$ beta dgdtp darcyKo a_oxygen
  5e-05 -0.0004 100000000.0 -1.0
*SELECT_DISCRETIZATION
power_law
*TRACK_ENERGY_BASED_FREE_SURFACE
$ lambda1 lambda2 surftens maxiter_energy tol_energy maxiter_bisect tol_bisect urf
  -100000.0 100000.0 1.8 30.0 1e-06 40.0 1e-18 0.5
*MESH_FILE
g_freesurf_mesh.k
*SINGLE_TRACK_TOOL
$ lasertime xstart ystart scanvel
  1.0 0.00021600000000000002 0.00021 1.0
