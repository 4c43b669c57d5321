! ISO_C_BINDING front end of libsalgpu.so for the reference's Fortran drivers.
!
! Drop-in for fast_sum_module (fast_sum_module.f90:291-332) and for the three
! mom6_fast_sum_module entry points (mom6_fast_sum_module.f90:33-192): the
! subroutines below keep their names, argument lists and intent(inout)
! accumulation, so code.f90 and mom6_code.f90 change only their `use` lines
! (fast_sum_module / mom6_fast_sum_module -> salgpu_mod).  No set-up call is
! needed: each call passes its arguments to the library, which hashes the
! set-up ones (coordinates, areas, panels, list, degree) and reuses the device
! grid it built for the same contents.
!
! cube_panel has allocatable components and interaction_pair is not bind(C),
! so both are flattened here on every call.  The panels go without their
! points_inside arrays (the library rebuilds the tree from the coordinates and
! checks it against the panels); only if that check fails (SAL_ETREE, e.g. a
! tree refined past its threshold by identical points) are points_inside
! flattened and the call repeated.
!
! Optional namelist group, read once from namelist.nml next to &params:
!   &gpu_params form = 0 (reference arithmetic) | 1 (accurate CP/CC),
!               mom6_mode = 1 (reference's transposed weights) | 2 (correct) /
!
! Build (where a Fortran compiler exists):
!   gfortran -O2 -c salgpu_mod.f90   (after tree_module.f90)
!   link with -L<repo>/sal-fort_b200/salgpu -lsalgpu -lstdc++ -lgomp
MODULE SALGPU_MOD
    use iso_c_binding
    use tree_module, only: cube_panel, interaction_pair
    implicit none
    private
    public :: fast_sum, proxy_source_compute, pc_compute, pp_compute, salgpu_read

    integer(c_int), parameter :: SAL_OK = 0, SAL_ETREE = -6

    interface
        integer(c_int) function sal_fast_sum(lon, lat, list, nlist, np, ints9, dbl7, pt_off, pt_idx, xs, ys, zs, &
                                             area, ssh, n, degree, rank, nproc) bind(C, name="sal_fast_sum")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
            real(c_double), intent(inout) :: lon(*), lat(*)
            integer(c_int32_t), intent(in) :: list(*), ints9(*)
            integer(c_int64_t), value :: nlist
            integer(c_int32_t), value :: np, n, degree, rank, nproc
            real(c_double), intent(in) :: dbl7(*), xs(*), ys(*), zs(*), area(*), ssh(*)
            integer(c_int64_t), intent(in) :: pt_off(*)
            type(c_ptr), value :: pt_idx
        end function
        integer(c_int) function sal_mom6_proxy_source_compute(w, np, ints9, dbl7, pt_off, pt_idx, points_panels, &
                nlev, xs, ys, zs, sshs, areas, degree, n) bind(C, name="sal_mom6_proxy_source_compute")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
            real(c_double), intent(inout) :: w(*)
            integer(c_int32_t), value :: np, nlev, degree, n
            integer(c_int32_t), intent(in) :: ints9(*), points_panels(*)
            real(c_double), intent(in) :: dbl7(*), xs(*), ys(*), zs(*), sshs(*), areas(*)
            integer(c_int64_t), intent(in) :: pt_off(*)
            type(c_ptr), value :: pt_idx
        end function
        integer(c_int) function sal_mom6_pc_compute(lon, lat, list, nlist, np, ints9, dbl7, pt_off, pt_idx, xs, ys, &
                zs, n, degree, w) bind(C, name="sal_mom6_pc_compute")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
            real(c_double), intent(inout) :: lon(*), lat(*)
            integer(c_int32_t), intent(in) :: list(*), ints9(*)
            integer(c_int64_t), value :: nlist
            integer(c_int32_t), value :: np, n, degree
            real(c_double), intent(in) :: dbl7(*), xs(*), ys(*), zs(*), w(*)
            integer(c_int64_t), intent(in) :: pt_off(*)
            type(c_ptr), value :: pt_idx
        end function
        integer(c_int) function sal_mom6_pp_compute(lon, lat, list, nlist, np, ints9, dbl7, pt_off, pt_idx, xs, ys, &
                zs, areas, sshs, e_xs, e_ys, e_zs, e_areas, e_sshs, n_extra, own) bind(C, name="sal_mom6_pp_compute")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
            real(c_double), intent(inout) :: lon(*), lat(*)
            integer(c_int32_t), intent(in) :: list(*), ints9(*)
            integer(c_int64_t), value :: nlist
            integer(c_int32_t), value :: np, n_extra, own
            real(c_double), intent(in) :: dbl7(*), xs(*), ys(*), zs(*), areas(*), sshs(*)
            real(c_double), intent(in) :: e_xs(*), e_ys(*), e_zs(*), e_areas(*), e_sshs(*)
            integer(c_int64_t), intent(in) :: pt_off(*)
            type(c_ptr), value :: pt_idx
        end function
        integer(c_int) function sal_dropin_config(form, mom6_mode) bind(C, name="sal_dropin_config")
            import :: c_int, c_int32_t
            integer(c_int32_t), value :: form, mom6_mode
        end function
        integer(c_int) function sal_read_values(path, count, out) bind(C, name="sal_read_values")
            import :: c_int, c_int64_t, c_double, c_char
            character(kind=c_char), intent(in) :: path(*)
            integer(c_int64_t), value :: count
            real(c_double), intent(out) :: out(*)
        end function
        type(c_ptr) function sal_last_error() bind(C, name="sal_last_error")
            import :: c_ptr
        end function
    end interface

    logical, save :: configured = .false.

    CONTAINS

    SUBROUTINE check(rc)
        integer(c_int), intent(in) :: rc
        character(kind=c_char), pointer :: msg(:)
        integer :: k
        IF (rc /= SAL_OK) THEN
            call c_f_pointer(sal_last_error(), msg, [512])
            k = 1
            DO WHILE (k < 512 .and. msg(k) /= c_null_char)
                k = k + 1
            END DO
            print *, 'salgpu error ', rc, ': ', msg(1:k-1)
            error stop
        END IF
    END SUBROUTINE

    ! Reads the optional &gpu_params group once (absent: reference behaviour).
    SUBROUTINE configure()
        integer :: form, mom6_mode, ios, u
        NAMELIST /gpu_params/ form, mom6_mode
        IF (configured) RETURN
        configured = .true.
        form = 0
        mom6_mode = 1
        open(newunit=u, file='namelist.nml', status='old', action='read', iostat=ios)
        IF (ios == 0) THEN
            read(u, nml=gpu_params, iostat=ios)
            close(u)
        END IF
        call check(sal_dropin_config(int(form, c_int32_t), int(mom6_mode, c_int32_t)))
    END SUBROUTINE

    ! The cube_panel array without points_inside (the sal_tree_import layout).
    SUBROUTINE flatten_panels(panels, ints9, dbl7, pt_off)
        type(cube_panel), intent(in) :: panels(:)
        integer(c_int32_t), allocatable, intent(out) :: ints9(:)
        real(c_double), allocatable, intent(out) :: dbl7(:)
        integer(c_int64_t), allocatable, intent(out) :: pt_off(:)
        integer :: k, np
        np = size(panels)
        allocate(ints9(9*np), dbl7(7*np), pt_off(np+1))
        pt_off(1) = 0
        DO k = 1, np
            ints9(9*(k-1)+1:9*k) = [panels(k)%level, merge(1, 0, panels(k)%is_leaf), panels(k)%id, &
                                    panels(k)%parent_panel, panels(k)%child_panel_1, panels(k)%child_panel_2, &
                                    panels(k)%child_panel_3, panels(k)%child_panel_4, panels(k)%face]
            dbl7(7*(k-1)+1:7*k) = [panels(k)%min_xi, panels(k)%mid_xi, panels(k)%max_xi, panels(k)%min_eta, &
                                   panels(k)%mid_eta, panels(k)%max_eta, panels(k)%radius]
            pt_off(k+1) = pt_off(k) + panels(k)%panel_point_count
        END DO
    END SUBROUTINE

    ! points_inside of every panel, concatenated (offsets pt_off).
    SUBROUTINE flatten_points(panels, pt_off, pt_idx)
        type(cube_panel), intent(in) :: panels(:)
        integer(c_int64_t), intent(in) :: pt_off(:)
        integer(c_int32_t), allocatable, target, intent(out) :: pt_idx(:)
        integer :: k
        allocate(pt_idx(max(pt_off(size(pt_off)), 1_c_int64_t)))
        DO k = 1, size(panels)
            IF (panels(k)%panel_point_count > 0) &
                pt_idx(pt_off(k)+1:pt_off(k+1)) = panels(k)%points_inside(1:panels(k)%panel_point_count)
        END DO
    END SUBROUTINE

    ! interaction_pair list as (target, source[, type]) int32 tuples.
    SUBROUTINE flatten_list(list, width, flat)
        type(interaction_pair), intent(in) :: list(:)
        integer, intent(in) :: width
        integer(c_int32_t), allocatable, intent(out) :: flat(:)
        integer :: i
        allocate(flat(max(width*size(list), 1)))
        DO i = 1, size(list)
            flat(width*(i-1)+1) = list(i)%index_target
            flat(width*(i-1)+2) = list(i)%index_source
            IF (width == 3) flat(width*i) = list(i)%interact_type
        END DO
    END SUBROUTINE

    ! Reads the first size(values) values of a one-value-per-line input file
    ! (or of its raw ".f64" form) with every host thread, in place of the
    ! drivers' list-directed read loops (code.f90:36-56):
    !     call salgpu_read('data-files/2313486_mpas_grid_x.csv', xs)
    SUBROUTINE salgpu_read(path, values)
        character(len=*), intent(in) :: path
        real(8), intent(out) :: values(:)
        call check(sal_read_values(trim(path)//c_null_char, int(size(values), c_int64_t), values))
    END SUBROUTINE

    ! fast_sum_module.f90:291-332, same arguments.
    SUBROUTINE fast_sum(sal_longrad, sal_latgrad, interaction_list, cube_panels, xs, ys, zs, area, ssh, point_count, &
                        interp_degree, rank, process_count)
        real(8), intent(in) :: xs(:), ys(:), zs(:), area(:), ssh(:)
        type(cube_panel), intent(in) :: cube_panels(:)
        type(interaction_pair), intent(in) :: interaction_list(:)
        integer, intent(in) :: point_count, interp_degree, rank, process_count
        real(8), intent(inout) :: sal_longrad(:), sal_latgrad(:)
        integer(c_int32_t), allocatable :: list(:), ints9(:)
        integer(c_int32_t), allocatable, target :: pt_idx(:)
        real(c_double), allocatable :: dbl7(:)
        integer(c_int64_t), allocatable :: pt_off(:)
        integer(c_int) :: rc
        call configure()
        call flatten_list(interaction_list, 3, list)
        call flatten_panels(cube_panels, ints9, dbl7, pt_off)
        rc = sal_fast_sum(sal_longrad, sal_latgrad, list, int(size(interaction_list), c_int64_t), &
                          int(size(cube_panels), c_int32_t), ints9, dbl7, pt_off, c_null_ptr, xs, ys, zs, area, ssh, &
                          int(point_count, c_int32_t), int(interp_degree, c_int32_t), int(rank, c_int32_t), &
                          int(process_count, c_int32_t))
        IF (rc == SAL_ETREE) THEN
            call flatten_points(cube_panels, pt_off, pt_idx)
            rc = sal_fast_sum(sal_longrad, sal_latgrad, list, int(size(interaction_list), c_int64_t), &
                              int(size(cube_panels), c_int32_t), ints9, dbl7, pt_off, c_loc(pt_idx), xs, ys, zs, &
                              area, ssh, int(point_count, c_int32_t), int(interp_degree, c_int32_t), &
                              int(rank, c_int32_t), int(process_count, c_int32_t))
        END IF
        call check(rc)
    END SUBROUTINE

    ! mom6_fast_sum_module.f90:33-74, same arguments.
    SUBROUTINE proxy_source_compute(proxy_source_weights, tree_panels, points_panels, xs, ys, zs, sshs, areas, &
                                    interp_degree, point_count)
        real(8), intent(out) :: proxy_source_weights(:)
        real(8), intent(in) :: xs(:), ys(:), zs(:), sshs(:), areas(:)
        type(cube_panel), intent(in) :: tree_panels(:)
        integer, intent(in) :: points_panels(:,:), interp_degree, point_count
        integer(c_int32_t), allocatable :: ints9(:), ppan(:)
        integer(c_int32_t), allocatable, target :: pt_idx(:)
        real(c_double), allocatable :: dbl7(:)
        integer(c_int64_t), allocatable :: pt_off(:)
        integer(c_int) :: rc
        call configure()
        call flatten_panels(tree_panels, ints9, dbl7, pt_off)
        ppan = reshape(points_panels(:, 1:point_count), [size(points_panels, 1) * point_count])
        rc = sal_mom6_proxy_source_compute(proxy_source_weights, int(size(tree_panels), c_int32_t), ints9, dbl7, &
                pt_off, c_null_ptr, ppan, int(size(points_panels, 1), c_int32_t), xs, ys, zs, sshs, areas, &
                int(interp_degree, c_int32_t), int(point_count, c_int32_t))
        IF (rc == SAL_ETREE) THEN
            call flatten_points(tree_panels, pt_off, pt_idx)
            rc = sal_mom6_proxy_source_compute(proxy_source_weights, int(size(tree_panels), c_int32_t), ints9, &
                    dbl7, pt_off, c_loc(pt_idx), ppan, int(size(points_panels, 1), c_int32_t), xs, ys, zs, sshs, &
                    areas, int(interp_degree, c_int32_t), int(point_count, c_int32_t))
        END IF
        call check(rc)
    END SUBROUTINE

    ! mom6_fast_sum_module.f90:153-174, same arguments.
    SUBROUTINE pc_compute(sal_longrad, sal_latgrad, pc_interaction_list, cube_panels, xs, ys, zs, interp_degree, &
                          proxy_weights)
        real(8), intent(in) :: xs(:), ys(:), zs(:), proxy_weights(:)
        type(interaction_pair), intent(in) :: pc_interaction_list(:)
        real(8), intent(inout) :: sal_longrad(:), sal_latgrad(:)
        type(cube_panel), intent(in) :: cube_panels(:)
        integer, intent(in) :: interp_degree
        integer(c_int32_t), allocatable :: list(:), ints9(:)
        integer(c_int32_t), allocatable, target :: pt_idx(:)
        real(c_double), allocatable :: dbl7(:)
        integer(c_int64_t), allocatable :: pt_off(:)
        integer(c_int) :: rc
        call configure()
        call flatten_list(pc_interaction_list, 2, list)
        call flatten_panels(cube_panels, ints9, dbl7, pt_off)
        rc = sal_mom6_pc_compute(sal_longrad, sal_latgrad, list, int(size(pc_interaction_list), c_int64_t), &
                int(size(cube_panels), c_int32_t), ints9, dbl7, pt_off, c_null_ptr, xs, ys, zs, &
                int(size(xs), c_int32_t), int(interp_degree, c_int32_t), proxy_weights)
        IF (rc == SAL_ETREE) THEN
            call flatten_points(cube_panels, pt_off, pt_idx)
            rc = sal_mom6_pc_compute(sal_longrad, sal_latgrad, list, int(size(pc_interaction_list), c_int64_t), &
                    int(size(cube_panels), c_int32_t), ints9, dbl7, pt_off, c_loc(pt_idx), xs, ys, zs, &
                    int(size(xs), c_int32_t), int(interp_degree, c_int32_t), proxy_weights)
        END IF
        call check(rc)
    END SUBROUTINE

    ! mom6_fast_sum_module.f90:177-192, same arguments (one rank: the e_*
    ! halo arrays of other ranks' points are empty).
    SUBROUTINE pp_compute(sal_longrad, sal_latgrad, pp_interaction_list, cube_panels, xs, ys, zs, areas, sshs, e_xs, &
                          e_ys, e_zs, e_areas, e_sshs, own_points)
        real(8), intent(inout) :: sal_longrad(:), sal_latgrad(:)
        type(interaction_pair), intent(in) :: pp_interaction_list(:)
        type(cube_panel), intent(in) :: cube_panels(:)
        real(8), intent(in) :: xs(:), ys(:), zs(:), areas(:), sshs(:), e_xs(:), e_ys(:), e_zs(:), e_areas(:), e_sshs(:)
        integer, intent(in) :: own_points
        integer(c_int32_t), allocatable :: list(:), ints9(:)
        integer(c_int32_t), allocatable, target :: pt_idx(:)
        real(c_double), allocatable :: dbl7(:)
        integer(c_int64_t), allocatable :: pt_off(:)
        real(c_double) :: none(1)
        integer(c_int) :: rc
        call configure()
        none = 0
        call flatten_list(pp_interaction_list, 2, list)
        call flatten_panels(cube_panels, ints9, dbl7, pt_off)
        IF (size(e_xs) > 0) THEN
            rc = sal_mom6_pp_compute(sal_longrad, sal_latgrad, list, int(size(pp_interaction_list), c_int64_t), &
                    int(size(cube_panels), c_int32_t), ints9, dbl7, pt_off, c_null_ptr, xs, ys, zs, areas, sshs, &
                    e_xs, e_ys, e_zs, e_areas, e_sshs, int(size(e_xs), c_int32_t), int(own_points, c_int32_t))
        ELSE
            rc = sal_mom6_pp_compute(sal_longrad, sal_latgrad, list, int(size(pp_interaction_list), c_int64_t), &
                    int(size(cube_panels), c_int32_t), ints9, dbl7, pt_off, c_null_ptr, xs, ys, zs, areas, sshs, &
                    none, none, none, none, none, 0_c_int32_t, int(own_points, c_int32_t))
        END IF
        IF (rc == SAL_ETREE) THEN
            call flatten_points(cube_panels, pt_off, pt_idx)
            rc = sal_mom6_pp_compute(sal_longrad, sal_latgrad, list, int(size(pp_interaction_list), c_int64_t), &
                    int(size(cube_panels), c_int32_t), ints9, dbl7, pt_off, c_loc(pt_idx), xs, ys, zs, areas, &
                    sshs, none, none, none, none, none, 0_c_int32_t, int(own_points, c_int32_t))
        END IF
        call check(rc)
    END SUBROUTINE
END MODULE
