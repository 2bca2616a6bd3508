!> ISO_C_BINDING interface of the Fortran host to the B200 step library
!> (include/ibisco_gpu.h).  Add this file to the reference's SOURCES before
!> main.F90 and link with -L<dir> -libisco_b200 -lcudart -lstdc++.
!>
!> The derived types mirror ibg_desc and ibg_obs field by field (BIND(C)
!> gives them the C struct layout).  IBG_DESC_FROM_VAR fills the descriptor
!> from MODULE VAR after the setup phase of main.F90 (lines 107-237) has run;
!> IBG_LOOP replaces the body of NEW_LOOP.F90:26-153 / MTS_LOOP.f90:24-53:
!> the step runs on the GPU, while AVERAGE, WRITETRJ and OUTPUT stay on the
!> host and read the observables the library returns.
!>
!> C_LOC needs TARGET or POINTER: every array used here is a POINTER in
!> module_var.F90 except BOND_TYPE_LABEL, ANGLE_TYPE_LABEL,
!> TORSION_TYPE_LABEL and OOP_TYPE_LABEL (module_var.F90:126-127), whose
!> declarations need ", TARGET" added.
MODULE IBISCO_GPU
  USE, INTRINSIC :: ISO_C_BINDING
  IMPLICIT NONE

  INTEGER(C_INT), PARAMETER :: IBG_PREC_FP32_FIXED = 0, IBG_PREC_FP64_PLAIN = 1
  INTEGER(C_INT), PARAMETER :: IBG_VS_COM_FIXED = 0, IBG_VS_COM_REFERENCE = 1
  INTEGER(C_INT), PARAMETER :: IBG_LIST_AUTO = -1, IBG_LIST_PER_PARTICLE = 0, IBG_LIST_PER_SLICE = 1

  TYPE, BIND(C) :: IBG_DESC_T
     INTEGER(C_INT) :: natoms, nvirta, nitems, ntype
     INTEGER(C_INT) :: numatoms, numbeads, ncoarse
     INTEGER(C_INT) :: ensemble, nupdate, halt_drift, nmts, ibrdescr, maxnab
     REAL(C_FLOAT) :: dt, fac, pfac, temp_in, pressure
     REAL(C_FLOAT) :: mktemp, mktemp_atom, mktemp_bead
     REAL(C_FLOAT) :: rcut_atom, rcutsq_atom, rlist_atom
     REAL(C_FLOAT) :: rcut_bead, rcutsq_bead, rlist_bead
     TYPE(C_PTR) :: mass, invmass, itype, type_label, atom, bead
     TYPE(C_PTR) :: nbonds, jbond
     INTEGER(C_INT) :: ld_bond
     TYPE(C_PTR) :: nijk, jangleijk, kangleijk
     INTEGER(C_INT) :: ld_angle
     TYPE(C_PTR) :: nijkl, jtorijkl, ktorijkl, ltorijkl
     INTEGER(C_INT) :: ld_torsion
     TYPE(C_PTR) :: noopijkl, joopijkl, koopijkl, loopijkl
     INTEGER(C_INT) :: ld_oop
     TYPE(C_PTR) :: connections, connected_to
     INTEGER(C_INT) :: ld_conn
     TYPE(C_PTR) :: ibondt, inbondt, iangt, itort, ioopt
     TYPE(C_PTR) :: bond_type_label, angle_type_label, torsion_type_label, oop_type_label
     INTEGER(C_INT) :: nbtype, natype, nttype, nnbtype, notype
     INTEGER(C_INT) :: ld_b, ld_a, ld_t, ld_nb, ld_o
     TYPE(C_PTR) :: ndatb, binb, rbond, bond_pot, bond_force
     TYPE(C_PTR) :: ndatan, bina, angle, bend_pot, bend_force
     TYPE(C_PTR) :: ndatt, bint, angle_tor, tor_pot, tor_force
     TYPE(C_PTR) :: ndatnb, binnb, rnbond, nbond_pot, nbond_force
     TYPE(C_PTR) :: ndato, bino, angle_oop, oop_pot, oop_force
     INTEGER(C_INT) :: ld_vs, vs_maxatoms
     TYPE(C_PTR) :: vitype, virt_center, virt_numatoms, virt_atm_ind
     TYPE(C_PTR) :: virt_invmass, virt_masscoeff
  END TYPE IBG_DESC_T

  TYPE, BIND(C) :: IBG_OBS_T
     REAL(C_DOUBLE) :: ek(2), temp, temp_atom, temp_bead
     REAL(C_DOUBLE) :: v_nb(3), v_bond(3), v_angle(3), v_torsion(3), v_oop(3)
     REAL(C_DOUBLE) :: pt(6), box(3)
     INTEGER(C_LONG_LONG) :: bond_overext, cell_clamps
     INTEGER(C_INT) :: step, status
  END TYPE IBG_OBS_T

  INTERFACE
     INTEGER(C_INT) FUNCTION ibg_create(d, precision, ctx) BIND(C, NAME='ibg_create')
       IMPORT :: C_INT, C_PTR, IBG_DESC_T
       TYPE(IBG_DESC_T), INTENT(IN) :: d
       INTEGER(C_INT), VALUE :: precision
       TYPE(C_PTR), INTENT(OUT) :: ctx
     END FUNCTION ibg_create

     !> Verlet-list form of the FP32 path: automatic (-1, the default), a
     !> list per particle (0) or per slice of four slots (1); before
     !> ibg_set_state.
     INTEGER(C_INT) FUNCTION ibg_set_list_form(ctx, form) BIND(C, NAME='ibg_set_list_form')
       IMPORT :: C_PTR, C_INT
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT), VALUE :: form
     END FUNCTION ibg_set_list_form

     !> Centre-of-mass virtual sites as VIRTUAL_DEF.f90 computes them (1) or
     !> each at its centre of mass (0, the default); before ibg_set_state.
     INTEGER(C_INT) FUNCTION ibg_set_vsite_com(ctx, form) BIND(C, NAME='ibg_set_vsite_com')
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT), VALUE :: form
     END FUNCTION ibg_set_vsite_com

     INTEGER(C_INT) FUNCTION ibg_set_state(ctx, sxyz, vxyz, box) BIND(C, NAME='ibg_set_state')
       IMPORT :: C_INT, C_PTR, C_FLOAT
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_FLOAT), INTENT(IN) :: sxyz(*), vxyz(*), box(3)
     END FUNCTION ibg_set_state

     INTEGER(C_INT) FUNCTION ibg_step(ctx, step, obs) BIND(C, NAME='ibg_step')
       IMPORT :: C_INT, C_PTR, IBG_OBS_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT), VALUE :: step
       TYPE(IBG_OBS_T), INTENT(OUT) :: obs
     END FUNCTION ibg_step

     INTEGER(C_INT) FUNCTION ibg_run(ctx, first, nsteps, per_step) BIND(C, NAME='ibg_run')
       IMPORT :: C_INT, C_PTR, IBG_OBS_T
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT), VALUE :: first, nsteps
       TYPE(IBG_OBS_T), INTENT(OUT) :: per_step(*)
     END FUNCTION ibg_run

     INTEGER(C_INT) FUNCTION ibg_get_state(ctx, sxyz, rxyz, vxyz, fxyz) BIND(C, NAME='ibg_get_state')
       IMPORT :: C_INT, C_PTR, C_FLOAT
       TYPE(C_PTR), VALUE :: ctx
       REAL(C_FLOAT), INTENT(OUT) :: sxyz(*), rxyz(*), vxyz(*), fxyz(*)
     END FUNCTION ibg_get_state

     INTEGER(C_INT) FUNCTION ibg_get_neighbour_list(ctx, which, list, maxnab, nnebs) &
          BIND(C, NAME='ibg_get_neighbour_list')
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT), VALUE :: which, maxnab
       INTEGER(C_INT), INTENT(OUT) :: list(*), nnebs(*)
     END FUNCTION ibg_get_neighbour_list

     TYPE(C_PTR) FUNCTION ibg_last_error(ctx) BIND(C, NAME='ibg_last_error')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ctx
     END FUNCTION ibg_last_error

     SUBROUTINE ibg_destroy(ctx) BIND(C, NAME='ibg_destroy')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ctx
     END SUBROUTINE ibg_destroy

     INTEGER(C_SIZE_T) FUNCTION c_strlen(s) BIND(C, NAME='strlen')
       IMPORT :: C_SIZE_T, C_PTR
       TYPE(C_PTR), VALUE :: s
     END FUNCTION c_strlen
  END INTERFACE

CONTAINS

  !> ibg_desc from MODULE VAR, after BUILD_CONNECTIVITY/RDVIRTBONDS (main.F90:210-216).
  SUBROUTINE IBG_DESC_FROM_VAR(D)
    USE VAR
    TYPE(IBG_DESC_T), INTENT(OUT) :: D
    D%natoms = NATOMS; D%nvirta = NVIRTA; D%nitems = NITEMS; D%ntype = NTYPE
    D%numatoms = NUMATOMS; D%numbeads = NUMBEADS; D%ncoarse = NCOARSE
    D%ensemble = ENSEMBLE; D%nupdate = NUPDATE; D%halt_drift = HALT_DRIFT
    D%nmts = NMTS; D%ibrdescr = IBRDESCR; D%maxnab = MAXNAB_ATOM
    D%dt = DT; D%fac = FAC; D%pfac = PFAC; D%temp_in = TEMP_IN; D%pressure = PRESSURE
    D%mktemp = MKTEMP; D%mktemp_atom = MKTEMP_ATOM; D%mktemp_bead = MKTEMP_BEAD
    D%rcut_atom = RCUT_ATOM; D%rcutsq_atom = RCUTSQ_ATOM; D%rlist_atom = RLIST_ATOM
    D%rcut_bead = RCUT_BEAD; D%rcutsq_bead = RCUTSQ_BEAD; D%rlist_bead = RLIST_BEAD
    D%mass = C_LOC(MASS); D%invmass = C_LOC(INVMASS)
    D%itype = C_LOC(ITYPE); D%type_label = C_LOC(TYPE_LABEL)
    D%atom = C_NULL_PTR; D%bead = C_NULL_PTR
    IF (NUMATOMS > 0) D%atom = C_LOC(ATOM)
    IF (NCOARSE > 0) D%bead = C_LOC(BEAD)
    D%nbonds = C_LOC(NBONDS); D%jbond = C_LOC(JBOND); D%ld_bond = SIZE(JBOND, 1)
    D%nijk = C_LOC(NIJK); D%jangleijk = C_LOC(JANGLEIJK); D%kangleijk = C_LOC(KANGLEIJK)
    D%ld_angle = SIZE(JANGLEIJK, 1)
    D%nijkl = C_LOC(NIJKL); D%jtorijkl = C_LOC(JTORIJKL); D%ktorijkl = C_LOC(KTORIJKL)
    D%ltorijkl = C_LOC(LTORIJKL); D%ld_torsion = SIZE(JTORIJKL, 1)
    D%noopijkl = C_LOC(NOOPIJKL); D%joopijkl = C_LOC(JOOPIJKL); D%koopijkl = C_LOC(KOOPIJKL)
    D%loopijkl = C_LOC(LOOPIJKL); D%ld_oop = SIZE(JOOPIJKL, 1)
    D%connections = C_LOC(CONNECTIONS); D%connected_to = C_LOC(CONNECTED_TO)
    D%ld_conn = SIZE(CONNECTED_TO, 1)
    D%ibondt = C_LOC(IBONDT); D%inbondt = C_LOC(INBONDT); D%iangt = C_LOC(IANGT)
    D%itort = C_LOC(ITORT); D%ioopt = C_LOC(IOOPT)
    D%nbtype = NBTYPE; D%natype = NATYPE; D%nttype = NTTYPE; D%nnbtype = NNBTYPE; D%notype = NOTYPE
    D%bond_type_label = C_NULL_PTR; D%angle_type_label = C_NULL_PTR
    D%torsion_type_label = C_NULL_PTR; D%oop_type_label = C_NULL_PTR
    D%ld_b = 0; D%ld_a = 0; D%ld_t = 0; D%ld_o = 0
    D%ndatb = C_NULL_PTR; D%binb = C_NULL_PTR; D%rbond = C_NULL_PTR; D%bond_pot = C_NULL_PTR; D%bond_force = C_NULL_PTR
    D%ndatan = C_NULL_PTR; D%bina = C_NULL_PTR; D%angle = C_NULL_PTR; D%bend_pot = C_NULL_PTR; D%bend_force = C_NULL_PTR
    D%ndatt = C_NULL_PTR; D%bint = C_NULL_PTR; D%angle_tor = C_NULL_PTR; D%tor_pot = C_NULL_PTR; D%tor_force = C_NULL_PTR
    D%ndato = C_NULL_PTR; D%bino = C_NULL_PTR; D%angle_oop = C_NULL_PTR; D%oop_pot = C_NULL_PTR; D%oop_force = C_NULL_PTR
    D%vitype = C_NULL_PTR; D%virt_center = C_NULL_PTR; D%virt_numatoms = C_NULL_PTR
    D%virt_atm_ind = C_NULL_PTR; D%virt_invmass = C_NULL_PTR; D%virt_masscoeff = C_NULL_PTR
    IF (NBTYPE > 0) THEN
       D%bond_type_label = C_LOC(BOND_TYPE_LABEL)
       D%ndatb = C_LOC(NDATB); D%binb = C_LOC(BINB); D%rbond = C_LOC(RBOND)
       D%bond_pot = C_LOC(BOND_POT); D%bond_force = C_LOC(BOND_FORCE); D%ld_b = SIZE(BOND_FORCE, 2)
    END IF
    IF (NATYPE > 0) THEN
       D%angle_type_label = C_LOC(ANGLE_TYPE_LABEL)
       D%ndatan = C_LOC(NDATAN); D%bina = C_LOC(BINA); D%angle = C_LOC(ANGLE)
       D%bend_pot = C_LOC(BEND_POT); D%bend_force = C_LOC(BEND_FORCE); D%ld_a = SIZE(BEND_FORCE, 2)
    END IF
    IF (NTTYPE > 0) THEN
       D%torsion_type_label = C_LOC(TORSION_TYPE_LABEL)
       D%ndatt = C_LOC(NDATT); D%bint = C_LOC(BINT); D%angle_tor = C_LOC(ANGLE_TOR)
       D%tor_pot = C_LOC(TOR_POT); D%tor_force = C_LOC(TOR_FORCE); D%ld_t = SIZE(TOR_FORCE, 2)
    END IF
    IF (NOTYPE > 0) THEN
       D%oop_type_label = C_LOC(OOP_TYPE_LABEL)
       D%ndato = C_LOC(NDATO); D%bino = C_LOC(BINO); D%angle_oop = C_LOC(ANGLE_OOP)
       D%oop_pot = C_LOC(OOP_POT); D%oop_force = C_LOC(OOP_FORCE); D%ld_o = SIZE(OOP_FORCE, 2)
    END IF
    D%ndatnb = C_LOC(NDATNB); D%binnb = C_LOC(BINNB); D%rnbond = C_LOC(RNBOND)
    D%nbond_pot = C_LOC(NBOND_POT); D%nbond_force = C_LOC(NBOND_FORCE); D%ld_nb = SIZE(NBOND_FORCE, 1)
    D%ld_vs = 0; D%vs_maxatoms = 0
    IF (NVIRTA > 0) THEN
       D%vitype = C_LOC(VITYPE); D%virt_center = C_LOC(VIRT_CENTER)
       D%virt_numatoms = C_LOC(VIRT_NUMATOMS); D%virt_atm_ind = C_LOC(VIRT_ATM_IND)
       D%ld_vs = SIZE(VIRT_ATM_IND, 1); D%vs_maxatoms = SIZE(VIRT_ATM_IND, 2)
       D%virt_invmass = C_LOC(VIRT_INVMASS); D%virt_masscoeff = C_LOC(VIRT_MASSCOEFF)
    END IF
  END SUBROUTINE IBG_DESC_FROM_VAR

  !> Observables of one step into the MODULE VAR scalars AVERAGE/OUTPUT read.
  SUBROUTINE IBG_OBS_TO_VAR(O)
    USE VAR
    TYPE(IBG_OBS_T), INTENT(IN) :: O
    EK = O%ek
    TEMP = REAL(O%temp, 4); TEMP_ATOM = REAL(O%temp_atom, 4); TEMP_BEAD = REAL(O%temp_bead, 4)
    V_NB = O%v_nb; V_BOND = O%v_bond; V_ANGLE = O%v_angle
    V_TORSION = O%v_torsion; V_OOP = O%v_oop
    PT11 = REAL(O%pt(1), 4); PT22 = REAL(O%pt(2), 4); PT33 = REAL(O%pt(3), 4)
    PT12 = REAL(O%pt(4), 4); PT13 = REAL(O%pt(5), 4); PT23 = REAL(O%pt(6), 4)
    BOX = REAL(O%box, 4)
    BOXINV = 1.0 / BOX
    BOX2 = BOX / 2.0
    VOLUME = BOX(1) * BOX(2) * BOX(3)
    INV_VOLUME = 1.0 / VOLUME
  END SUBROUTINE IBG_OBS_TO_VAR

  !> Replacement of the MD loop: one library step per STEP, host-side
  !> AVERAGE every step and WRITETRJ/OUTPUT every NTRJ steps with the state
  !> copied back first.  Any library failure sets ISTOP and ends the loop,
  !> as the reference's fatal STOPs do.
  SUBROUTINE IBG_LOOP(PRECISION)
    USE VAR
    INTEGER(C_INT), INTENT(IN) :: PRECISION
    TYPE(IBG_DESC_T) :: D
    TYPE(IBG_OBS_T) :: O
    TYPE(C_PTR) :: CTX
    INTEGER(C_INT) :: RC
    INTEGER :: STEP
    CALL IBG_DESC_FROM_VAR(D)
    RC = ibg_create(D, PRECISION, CTX)
    IF (RC /= 0) THEN
       WRITE(1, *) 'ibg_create failed with status ', RC
       ISTOP = 1
       RETURN
    END IF
    RC = ibg_set_state(CTX, SXYZ, VXYZ, BOX)
    DO STEP = 1, NSTEP
       IF (RC /= 0) EXIT
       RC = ibg_step(CTX, STEP, O)
       IF (RC /= 0) EXIT
       CALL IBG_OBS_TO_VAR(O)
       IF (MOD(STEP, NTRJ) == 0) THEN
          RC = ibg_get_state(CTX, SXYZ, RXYZ, VXYZ, FXYZ)
          IF (RC /= 0) EXIT
       END IF
       CALL AVERAGE()
       IF (MOD(STEP, NTRJ) == 0) THEN
          CALL WRITETRJ(STEP)
          CALL OUTPUT(STEP)
       END IF
    END DO
    IF (RC /= 0) THEN
       CALL REPORT_ERROR(CTX, RC)
       ISTOP = 1
    END IF
    CALL ibg_destroy(CTX)
  END SUBROUTINE IBG_LOOP

  SUBROUTINE REPORT_ERROR(CTX, RC)
    TYPE(C_PTR), INTENT(IN) :: CTX
    INTEGER(C_INT), INTENT(IN) :: RC
    TYPE(C_PTR) :: P
    CHARACTER(KIND=C_CHAR), POINTER :: S(:)
    INTEGER :: N
    P = ibg_last_error(CTX)
    N = INT(c_strlen(P))
    CALL C_F_POINTER(P, S, [N])
    WRITE(1, *) 'B200 step failed with status ', RC, ': ', S(1:N)
  END SUBROUTINE REPORT_ERROR

END MODULE IBISCO_GPU
