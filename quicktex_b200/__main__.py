from quicktex_b200.cli import main

if __name__ == "__main__":
    main()
