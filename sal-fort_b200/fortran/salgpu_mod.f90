! ISO_C_BINDING front end of libsalgpu.so for the reference's Fortran drivers.
!
! Drop-in for fast_sum_module (fast_sum_module.f90:291-332) and for the three
! mom6_fast_sum_module entry points (mom6_fast_sum_module.f90:33-192): the
! subroutines below keep their names, argument lists and intent(inout)
! accumulation, so code.f90 and mom6_code.f90 change only their `use` lines.
! The device grid is built on the first call and cached; later calls with the
! same tree and list reuse it.
!
! Build (where a Fortran compiler exists):
!   gfortran -O2 -c salgpu_mod.f90   (after tree_module.f90)
!   link with -L<repo>/sal-fort_b200/salgpu -lsalgpu -lstdc++ -lgomp
MODULE SALGPU_MOD
    use iso_c_binding
    use tree_module, only: cube_panel, interaction_pair
    implicit none

    integer(c_int), parameter :: SAL_OK = 0
    integer(c_int), parameter :: SAL_MODE_DTT = 0, SAL_MODE_STT_REF_COMPAT = 1, SAL_MODE_STT_CORRECT = 2
    integer(c_int), parameter :: SAL_FORM_REF = 0, SAL_FORM_ACCURATE = 1

    type, bind(C) :: sal_grid_desc
        integer(c_int32_t) :: point_count
        type(c_ptr) :: xs, ys, zs, areas
        integer(c_int32_t) :: interp_degree, mode
        type(c_ptr) :: list
        integer(c_int64_t) :: list_count
        type(c_ptr) :: pc_list
        integer(c_int64_t) :: pc_count
        type(c_ptr) :: pp_list
        integer(c_int64_t) :: pp_count
        integer(c_int32_t) :: max_fields, device
    end type

    interface
        integer(c_int) function sal_tree_import(np, ints9, dbl7, pt_off, pt_idx, n, xs, ys, zs, tree) &
                bind(C, name="sal_tree_import")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
            integer(c_int32_t), value :: np, n
            integer(c_int32_t), intent(in) :: ints9(*), pt_idx(*)
            real(c_double), intent(in) :: dbl7(*), xs(*), ys(*), zs(*)
            integer(c_int64_t), intent(in) :: pt_off(*)
            type(c_ptr), intent(out) :: tree
        end function
        integer(c_int) function sal_grid_create(tree, desc, grid) bind(C, name="sal_grid_create")
            import :: c_int, c_ptr, sal_grid_desc
            type(c_ptr), value :: tree
            type(sal_grid_desc), intent(in) :: desc
            type(c_ptr), intent(out) :: grid
        end function
        integer(c_int) function sal_fast_sum_host(grid, ssh, lon, lat, form) bind(C, name="sal_fast_sum_host")
            import :: c_int, c_int32_t, c_double, c_ptr
            type(c_ptr), value :: grid
            real(c_double), intent(in) :: ssh(*)
            real(c_double), intent(inout) :: lon(*), lat(*)
            integer(c_int32_t), value :: form
        end function
        integer(c_int) function sal_proxy_source_compute_host(grid, sshs, w) &
                bind(C, name="sal_proxy_source_compute_host")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: grid
            real(c_double), intent(in) :: sshs(*)
            real(c_double), intent(inout) :: w(*)
        end function
        integer(c_int) function sal_pc_compute_host(grid, w, sx, sy) bind(C, name="sal_pc_compute_host")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: grid
            real(c_double), intent(in) :: w(*)
            real(c_double), intent(inout) :: sx(*), sy(*)
        end function
        integer(c_int) function sal_pp_compute_host(grid, sshs, sx, sy) bind(C, name="sal_pp_compute_host")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: grid
            real(c_double), intent(in) :: sshs(*)
            real(c_double), intent(inout) :: sx(*), sy(*)
        end function
        type(c_ptr) function sal_last_error() bind(C, name="sal_last_error")
            import :: c_ptr
        end function
    end interface

    type(c_ptr), save :: dtt_grid = c_null_ptr, stt_grid = c_null_ptr
    integer, save :: dtt_key(3) = -1, stt_key(3) = -1

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

    ! Flattens a cube_panel array (allocatable components, not interoperable)
    ! into the sal_tree_import layout and imports it.
    SUBROUTINE import_tree(panels, xs, ys, zs, point_count, tree)
        type(cube_panel), intent(in) :: panels(:)
        real(8), intent(in), target :: xs(:), ys(:), zs(:)
        integer, intent(in) :: point_count
        type(c_ptr), intent(out) :: tree
        integer(c_int32_t), allocatable :: ints9(:), pt_idx(:)
        real(c_double), allocatable :: dbl7(:)
        integer(c_int64_t), allocatable :: pt_off(:)
        integer :: k, np, total
        np = size(panels)
        allocate(ints9(9*np), dbl7(7*np), pt_off(np+1))
        total = 0
        DO k = 1, np
            total = total + panels(k)%panel_point_count
        END DO
        allocate(pt_idx(max(total, 1)))
        pt_off(1) = 0
        DO k = 1, np
            ints9(9*(k-1)+1:9*k) = [panels(k)%level, merge(1, 0, panels(k)%is_leaf), panels(k)%id, &
                                    panels(k)%parent_panel, panels(k)%child_panel_1, panels(k)%child_panel_2, &
                                    panels(k)%child_panel_3, panels(k)%child_panel_4, panels(k)%face]
            dbl7(7*(k-1)+1:7*k) = [panels(k)%min_xi, panels(k)%mid_xi, panels(k)%max_xi, panels(k)%min_eta, &
                                   panels(k)%mid_eta, panels(k)%max_eta, panels(k)%radius]
            pt_off(k+1) = pt_off(k) + panels(k)%panel_point_count
            IF (panels(k)%panel_point_count > 0) &
                pt_idx(pt_off(k)+1:pt_off(k+1)) = panels(k)%points_inside(1:panels(k)%panel_point_count)
        END DO
        call check(sal_tree_import(int(np, c_int32_t), ints9, dbl7, pt_off, pt_idx, int(point_count, c_int32_t), &
                                   xs, ys, zs, tree))
    END SUBROUTINE

    ! fast_sum_module.f90:291-332, same arguments.
    SUBROUTINE fast_sum(sal_longrad, sal_latgrad, interaction_list, cube_panels, xs, ys, zs, area, ssh, point_count, &
                        interp_degree, rank, process_count)
        real(8), intent(in), target :: xs(:), ys(:), zs(:), area(:), ssh(:)
        type(cube_panel), intent(in) :: cube_panels(:)
        type(interaction_pair), intent(in) :: interaction_list(:)
        integer, intent(in) :: point_count, interp_degree, rank, process_count
        real(8), intent(inout) :: sal_longrad(:), sal_latgrad(:)
        integer(c_int32_t), allocatable, target :: flat(:)
        type(sal_grid_desc) :: d
        type(c_ptr) :: tree
        integer :: i, m
        IF (.not. c_associated(dtt_grid) .or. any(dtt_key /= [size(interaction_list), size(cube_panels), rank])) THEN
            allocate(flat(3*size(interaction_list)))
            m = 0
            DO i = 1, size(interaction_list)
                IF (MOD(i, process_count) == rank) THEN      ! fast_sum_module.f90:304
                    flat(3*m+1:3*m+3) = [interaction_list(i)%index_target, interaction_list(i)%index_source, &
                                         interaction_list(i)%interact_type]
                    m = m + 1
                END IF
            END DO
            call import_tree(cube_panels, xs, ys, zs, point_count, tree)
            d%point_count = point_count
            d%xs = c_loc(xs); d%ys = c_loc(ys); d%zs = c_loc(zs); d%areas = c_loc(area)
            d%interp_degree = interp_degree
            d%mode = SAL_MODE_DTT
            d%list = c_loc(flat); d%list_count = m
            d%pc_list = c_null_ptr; d%pc_count = 0; d%pp_list = c_null_ptr; d%pp_count = 0
            d%max_fields = 1; d%device = 0
            call check(sal_grid_create(tree, d, dtt_grid))
            dtt_key = [size(interaction_list), size(cube_panels), rank]
        END IF
        call check(sal_fast_sum_host(dtt_grid, ssh, sal_longrad, sal_latgrad, SAL_FORM_REF))
    END SUBROUTINE

    ! The MOM6 path needs its lists before the first solve: call this once after
    ! single_tree_traversal (mom6_code.f90:201), at one rank.
    SUBROUTINE salgpu_mom6_setup(tree_panels, pc_list, pp_list, xs, ys, zs, areas, point_count, interp_degree, &
                                 ref_compat)
        type(cube_panel), intent(in) :: tree_panels(:)
        type(interaction_pair), intent(in) :: pc_list(:), pp_list(:)
        real(8), intent(in), target :: xs(:), ys(:), zs(:), areas(:)
        integer, intent(in) :: point_count, interp_degree
        logical, intent(in) :: ref_compat
        integer(c_int32_t), allocatable, target :: a(:), b(:)
        type(sal_grid_desc) :: d
        type(c_ptr) :: tree
        integer :: i
        allocate(a(2*size(pc_list)), b(2*size(pp_list)))
        DO i = 1, size(pc_list)
            a(2*i-1:2*i) = [pc_list(i)%index_target, pc_list(i)%index_source]
        END DO
        DO i = 1, size(pp_list)
            b(2*i-1:2*i) = [pp_list(i)%index_target, pp_list(i)%index_source]
        END DO
        call import_tree(tree_panels, xs, ys, zs, point_count, tree)
        d%point_count = point_count
        d%xs = c_loc(xs); d%ys = c_loc(ys); d%zs = c_loc(zs); d%areas = c_loc(areas)
        d%interp_degree = interp_degree
        d%mode = merge(SAL_MODE_STT_REF_COMPAT, SAL_MODE_STT_CORRECT, ref_compat)
        d%list = c_null_ptr; d%list_count = 0
        d%pc_list = c_loc(a); d%pc_count = size(pc_list)
        d%pp_list = c_loc(b); d%pp_count = size(pp_list)
        d%max_fields = 1; d%device = 0
        call check(sal_grid_create(tree, d, stt_grid))
    END SUBROUTINE

    ! mom6_fast_sum_module.f90:33-74 (points_panels and the tree are already in the grid).
    SUBROUTINE proxy_source_compute(proxy_source_weights, sshs)
        real(8), intent(inout) :: proxy_source_weights(:)
        real(8), intent(in) :: sshs(:)
        call check(sal_proxy_source_compute_host(stt_grid, sshs, proxy_source_weights))
    END SUBROUTINE

    ! mom6_fast_sum_module.f90:153-174.
    SUBROUTINE pc_compute(sal_longrad, sal_latgrad, proxy_weights)
        real(8), intent(inout) :: sal_longrad(:), sal_latgrad(:)
        real(8), intent(in) :: proxy_weights(:)
        call check(sal_pc_compute_host(stt_grid, proxy_weights, sal_longrad, sal_latgrad))
    END SUBROUTINE

    ! mom6_fast_sum_module.f90:177-192 at one rank.
    SUBROUTINE pp_compute(sal_longrad, sal_latgrad, sshs)
        real(8), intent(inout) :: sal_longrad(:), sal_latgrad(:)
        real(8), intent(in) :: sshs(:)
        call check(sal_pp_compute_host(stt_grid, sshs, sal_longrad, sal_latgrad))
    END SUBROUTINE
END MODULE
